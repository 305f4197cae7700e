// MPS reader. It accepts the language below and builds the same models, with the same error messages and the
// same first error, as the reference reader (src/mps.cpp), whose models the PDHG path consumes.
//
// Grammar. A file is a sequence of lines; a trailing '\r' is dropped, and blank lines and lines starting with '*'
// are skipped. A line starting with anything but a space or a tab is a section header: its first word names the
// section, its second (if any) is an argument. Every other line is a data line of the current section, split
// into whitespace-separated fields (free format) or, when the whole file fails in free format, into the fixed
// columns 2-3, 5-12, 15-22, 25-36, 40-47 and 50-61 (ROWS: 2-3, 5-12; BOUNDS: 2-3, 5-12, 15-22, 25-36).
//   NAME [name]                    the model's name
//   OBJSENSE [MIN|MAX|MINIMIZE|MAXIMIZE]  the sense, on the header or on the section's first data line
//   ROWS       type name           type N (the first is the objective, later ones are ignored), E, L or G
//   COLUMNS    col row value [row value]   entries; a column's lines are consecutive; a line
//              MARKER 'MARKER' 'INTORG'|'INTEND' opens or closes a block of integer columns
//   RHS        [set] row value [row value] right-hand sides; on the objective row, minus the objective constant
//   RANGES     [set] row value [row value] row ranges
//   BOUNDS     type [set] col [value]      LO UP FX FR MI PL BV LI UI
//   QUADOBJ | QMATRIX | QSECTION obj       col col value: quadratic objective terms (counted, then rejected
//                                          by the input gate); QCMATRIX or QSECTION of another row is an error
//   ENDATA                         ends the file (required)
// Only the first named RHS, RANGES and BOUNDS set is used. Numbers are [+-] digits [. digits] [(e|E|d|D) [+-]
// digits] with at least one mantissa digit and must be finite. A column's entries are sorted by row, entries of
// one row summed in file order and zero sums dropped. Row bounds: E rows b (a range R moves the upper bound to b
// + R for R >= 0, else the lower to b + R), L rows (b - |R| or -inf, b), G rows (b, b + |R| or +inf). A finite
// bound of magnitude >= 1e20 reads as infinite (and is counted). Columns default to [0, +inf); UP below 0 on a
// zero lower bound makes the lower bound -inf.
//
// Large COLUMNS and BOUNDS sections (free format, >= 2 MB) are tokenised on all host threads in line-aligned
// chunks and applied in file order, so the model and the first error reported do not depend on the thread count.
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <string_view>
#include <thread>
#include <unordered_set>

#include "host.hpp"

namespace taral {
namespace {

constexpr double kHuge = 1e20;  // |bound| >= 1e20 is infinite

// ------------------------------------------------------------------------------------------------------ lexing
bool digit(char c) { return c >= '0' && c <= '9'; }
bool blank(char c) { return c == ' ' || c == '\t'; }
bool space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }

// [+-] digits [. digits] [(e|E|d|D) [+-] digits], at least one mantissa digit, the whole token
bool plain_decimal(std::string_view s) {
    size_t i = 0;
    const size_t n = s.size();
    auto skip_sign = [&] {
        if (i < n && (s[i] == '+' || s[i] == '-')) ++i;
    };
    auto count_digits = [&] {
        const size_t from = i;
        while (i < n && digit(s[i])) ++i;
        return i - from;
    };
    skip_sign();
    size_t mantissa = count_digits();
    if (i < n && s[i] == '.') {
        ++i;
        mantissa += count_digits();
    }
    if (mantissa == 0) return false;
    if (i < n && (s[i] == 'e' || s[i] == 'E' || s[i] == 'd' || s[i] == 'D')) {
        ++i;
        skip_sign();
        if (count_digits() == 0) return false;
    }
    return i == n;
}

double parse_number(std::string_view s) {
    if (!plain_decimal(s)) throw ParseError("bad number '" + std::string(s) + "'");
    // a NUL-terminated copy with the Fortran exponent letters d / D read as E (on the stack for short tokens)
    char local[64];
    std::string heap;
    char* b = local;
    if (s.size() >= sizeof local) heap.resize(s.size() + 1), b = &heap[0];
    for (size_t k = 0; k < s.size(); ++k) b[k] = (s[k] == 'd' || s[k] == 'D') ? 'E' : s[k];
    b[s.size()] = '\0';
    const char* e = b + s.size();
    // from_chars rounds like strtod; text outside the double range goes to strtod for its overflow / underflow value
    double v = 0;
    const auto res = std::from_chars(b, e, v);
    if (res.ec != std::errc() || res.ptr != e) v = std::strtod(b, nullptr);
    if (!std::isfinite(v)) throw ParseError("number '" + std::string(s) + "' is not finite");
    return v;
}

// the fixed-column field [a, b) of a line, trimmed of blanks; empty when the line is shorter than a
std::string_view column_field(std::string_view line, size_t a, size_t b) {
    if (line.size() <= a) return {};
    std::string_view f = line.substr(a, b - a);
    while (!f.empty() && blank(f.front())) f.remove_prefix(1);
    while (!f.empty() && (blank(f.back()) || f.back() == '\r')) f.remove_suffix(1);
    return f;
}

enum class Section { None, ObjSense, Rows, Columns, Rhs, Ranges, Bounds, Quad };

using Fields = std::vector<std::string_view>;

void free_fields(std::string_view line, Fields& out) {
    out.clear();
    size_t p = 0;
    while (p < line.size()) {
        while (p < line.size() && space(line[p])) ++p;
        const size_t from = p;
        while (p < line.size() && !space(line[p])) ++p;
        if (p > from) out.push_back(line.substr(from, p - from));
    }
}

void fixed_fields(std::string_view line, Section sec, Fields& out) {
    out.clear();
    auto take = [&](size_t a, size_t b) { out.push_back(column_field(line, a, b)); };
    if (sec == Section::Rows) {
        take(1, 3), take(4, 12);
    } else if (sec == Section::Bounds) {
        take(1, 3), take(4, 12), take(14, 22);
        if (!column_field(line, 24, 36).empty()) take(24, 36);
    } else {
        take(4, 12), take(14, 22), take(24, 36);
        if (!column_field(line, 39, 47).empty()) take(39, 47), take(49, 61);
    }
}

// Lines of buf[pos, end) that carry data or a header: '\r' dropped, blank and comment lines skipped.
class LineCursor {
  public:
    LineCursor(const std::string& buf, size_t pos, size_t end) : buf_(buf), pos_(pos), end_(end) {}
    bool next(std::string_view& line) {
        while (pos_ < end_) {
            size_t nl = buf_.find('\n', pos_);
            if (nl == std::string::npos || nl > end_) nl = end_;
            std::string_view l(buf_.data() + pos_, nl - pos_);
            pos_ = nl + 1;
            if (!l.empty() && l.back() == '\r') l.remove_suffix(1);
            if (l.find_first_not_of(" \t") == std::string_view::npos || l[0] == '*') continue;
            line = l;
            return true;
        }
        return false;
    }
    size_t pos() const { return pos_; }
    void seek(size_t p) { pos_ = p; }

  private:
    const std::string& buf_;
    size_t pos_, end_;
};

bool is_header_line(std::string_view line) { return !blank(line[0]); }

// Byte offset of the first header line at or after pos (the end of the section that starts at pos).
size_t section_end(const std::string& buf, size_t pos) {
    LineCursor cur(buf, pos, buf.size());
    std::string_view line;
    while (cur.next(line))
        if (is_header_line(line)) return size_t(line.data() - buf.data());
    return buf.size();
}

// Line-aligned cut points of [b, e) into `parts` chunks.
std::vector<size_t> chunk_cuts(const std::string& buf, size_t b, size_t e, int parts) {
    std::vector<size_t> cut{b};
    for (int q = 1; q < parts; ++q) {
        const size_t want = std::max(b + (e - b) * size_t(q) / size_t(parts), cut.back());
        const size_t nl = buf.find('\n', want);
        cut.push_back(nl == std::string::npos || nl >= e ? e : nl + 1);
    }
    cut.push_back(e);
    return cut;
}

template <class Work>
void on_threads(int parts, Work work) {
    std::vector<std::thread> pool;
    for (int q = 1; q < parts; ++q) pool.emplace_back(work, q);
    work(0);
    for (std::thread& t : pool) t.join();
}

// ------------------------------------------------------------------------------------------------ name tables
// Name -> index: open addressing with linear probing, grown at half load. A slot is 8 bytes (the upper half of a
// 64-bit FNV-1a hash and the index), so a probe costs one cache line; a tag match is confirmed against the name of
// that index, a view into the file buffer (the buffer outlives the table).
class NameTable {
  public:
    explicit NameTable(size_t expect) { rehash(std::max<size_t>(64, next_pow2(2 * expect))); }
    const int* find(std::string_view k) const {
        const uint64_t h = hash(k);
        const uint32_t tag = uint32_t(h >> 32);
        for (size_t i = h & mask_;; i = (i + 1) & mask_) {
            const Slot& s = slot_[i];
            if (s.idx < 0) return nullptr;
            if (s.tag == tag && name_[size_t(s.idx)] == k) return &s.idx;
        }
    }
    bool contains(std::string_view k) const { return find(k) != nullptr; }
    // Adds k unless it is present (one probe sequence); returns -1 when added, else the index k already has.
    int add_if_absent(std::string_view k) {
        if (2 * (name_.size() + 1) > slot_.size()) rehash(2 * slot_.size());
        const uint64_t h = hash(k);
        const uint32_t tag = uint32_t(h >> 32);
        size_t i = h & mask_;
        for (;; i = (i + 1) & mask_) {
            const Slot& s = slot_[i];
            if (s.idx < 0) break;
            if (s.tag == tag && name_[size_t(s.idx)] == k) return s.idx;
        }
        slot_[i] = {tag, int(name_.size())};
        name_.push_back(k);
        return -1;
    }

  private:
    struct Slot {
        uint32_t tag;
        int idx;
    };
    std::vector<Slot> slot_;
    std::vector<std::string_view> name_;
    size_t mask_ = 0;
    static size_t next_pow2(size_t x) {
        size_t p = 1;
        while (p < x) p <<= 1;
        return p;
    }
    static uint64_t hash(std::string_view k) {
        uint64_t h = 1469598103934665603ull;
        for (unsigned char c : k) h = (h ^ c) * 1099511628211ull;
        return h ^ (h >> 29);
    }
    void place(uint64_t h, int v) {
        size_t i = h & mask_;
        while (slot_[i].idx >= 0) i = (i + 1) & mask_;
        slot_[i] = {uint32_t(h >> 32), v};
    }
    void rehash(size_t size) {
        slot_.assign(size, Slot{0, -1});
        mask_ = size - 1;
        for (size_t v = 0; v < name_.size(); ++v) place(hash(name_[v]), int(v));
    }
};

// ------------------------------------------------------------------------------------------------ the model
enum class BoundKind { LO, UP, FX, FR, MI, PL, BV, LI, UI, Invalid };

BoundKind bound_kind(std::string_view t) {
    static const std::pair<std::string_view, BoundKind> kinds[] = {
        {"LO", BoundKind::LO}, {"UP", BoundKind::UP}, {"FX", BoundKind::FX}, {"FR", BoundKind::FR},
        {"MI", BoundKind::MI}, {"PL", BoundKind::PL}, {"BV", BoundKind::BV}, {"LI", BoundKind::LI},
        {"UI", BoundKind::UI}};
    for (const auto& k : kinds)
        if (k.first == t) return k.second;
    return BoundKind::Invalid;
}
bool bound_has_no_value(std::string_view t) { return t == "FR" || t == "MI" || t == "PL" || t == "BV"; }

constexpr int kObjectiveRow = -1;  // row references that are not constraint rows
constexpr int kIgnoredRow = -2;    // an N row after the first

// Accumulates the model from the records of the file, in file order. Names are views into the file buffer.
class ModelBuilder {
  public:
    explicit ModelBuilder(size_t file_bytes) : rows_(file_bytes / 512 + 16), cols_(file_bytes / 256 + 16) {}
    Model md;

    // --- ROWS
    void declare_row(std::string_view type, std::string_view name) {
        const char t = type.empty() ? '?' : char(std::toupper(static_cast<unsigned char>(type[0])));
        if (rows_.contains(name) || name == objective_ || ignored_rows_.count(name))
            throw ParseError("duplicate row name '" + std::string(name) + "'");
        if (t == 'N') {
            if (objective_.empty()) objective_ = std::string(name);
            else ignored_rows_.insert(name);
        } else if (t == 'E' || t == 'L' || t == 'G') {
            rows_.add_if_absent(name);
            md.row_names.emplace_back(name);
            row_kind_.push_back(t);
        } else {
            throw ParseError("bad row type " + std::string(type));
        }
    }
    const std::string& objective() const { return objective_; }
    // index of a constraint row, kObjectiveRow, kIgnoredRow; unknown names are an error
    int row(std::string_view name) const {
        if (const int* r = rows_.find(name)) return *r;
        if (name == objective_) return kObjectiveRow;
        if (ignored_rows_.count(name)) return kIgnoredRow;
        throw ParseError("unknown row '" + std::string(name) + "'");
    }

    // --- COLUMNS
    void integer_marker(bool opens) { in_integer_block_ = opens; }
    // The column named `name` becomes current (a new column unless it is the current one).
    void use_column(std::string_view name) {
        if (current_ >= 0 && name == current_name_) return;
        if (cols_.add_if_absent(name) >= 0)
            throw ParseError("column '" + std::string(name) + "' is listed in two separate blocks");
        close_column();
        current_ = int(md.col_names.size());
        current_name_ = name;
        md.col_names.emplace_back(name);
        md.cost.push_back(0);
        md.is_int.push_back(in_integer_block_ ? 1 : 0);
    }
    void add_entry(int row, double v) {  // into the current column
        if (row == kObjectiveRow) md.cost[size_t(current_)] += v;
        else if (row >= 0) pending_.push_back({row, v});
    }
    void reserve_entries(size_t entries, size_t columns) {
        md.row_idx.reserve(md.row_idx.size() + entries), md.val.reserve(md.val.size() + entries);
        md.col_names.reserve(md.col_names.size() + columns), md.cost.reserve(md.cost.size() + columns);
        md.is_int.reserve(md.is_int.size() + columns), md.col_ptr.reserve(md.col_ptr.size() + columns);
    }
    int column(std::string_view name) const {
        if (const int* c = cols_.find(name)) return *c;
        throw ParseError("unknown column '" + std::string(name) + "'");
    }
    const int* find_column(std::string_view name) const { return cols_.find(name); }

    // --- RHS / RANGES / BOUNDS sets: the first named set is used, lines of other sets are skipped
    static bool in_first_set(std::string& first, std::string_view name) {
        if (first.empty()) first = std::string(name);
        return first == name;
    }
    std::string rhs_set, range_set, bound_set;
    void set_rhs(int row, double v) {
        row_data();
        if (row == kObjectiveRow) md.obj_const = -v;
        else if (row >= 0) rhs_[size_t(row)] = v;
    }
    void set_range(int row, double v) {
        row_data();
        if (row >= 0) range_[size_t(row)] = v, has_range_[size_t(row)] = 1;
    }
    void row_data() {  // RHS / RANGES arrays, zero-filled on first use
        if (rhs_.size() < md.row_names.size()) {
            rhs_.resize(md.row_names.size(), 0.0);
            range_.resize(md.row_names.size(), 0.0);
            has_range_.resize(md.row_names.size(), 0);
        }
    }
    void column_bounds() {  // [0, +inf) for every column without bounds yet
        md.col_lo.resize(md.col_names.size(), 0.0);
        md.col_up.resize(md.col_names.size(), kInf);
    }
    void apply_bound(int j, std::string_view type, double v) {
        const BoundKind k = bound_kind(type);
        double& lo = md.col_lo[size_t(j)];
        double& up = md.col_up[size_t(j)];
        switch (k) {
            case BoundKind::LO: lo = v; break;
            case BoundKind::LI: md.is_int[size_t(j)] = 1, lo = v; break;
            case BoundKind::UI: md.is_int[size_t(j)] = 1; [[fallthrough]];
            case BoundKind::UP:
                up = v;
                if (v < 0 && lo == 0) lo = -kInf;
                break;
            case BoundKind::FX: lo = up = v; break;
            case BoundKind::FR: lo = -kInf, up = kInf; break;
            case BoundKind::MI: lo = -kInf; break;
            case BoundKind::PL: up = kInf; break;
            case BoundKind::BV: md.is_int[size_t(j)] = 1, lo = 0, up = 1; break;
            case BoundKind::Invalid: throw ParseError("unsupported bound type " + std::string(type));
        }
    }

    // --- quadratic objective: lower-triangle terms summed (a full matrix lists each off-diagonal term twice)
    bool quad_full = false;
    void quad_term(int a, int b, double v) {
        if (quad_full && a < b) return;
        quad_[{std::max(a, b), std::min(a, b)}] += v;
    }

    // --- end of file
    Model finish() {
        close_column();
        for (const auto& kv : quad_)
            if (kv.second != 0) ++md.n_quadratic;
        if (objective_.empty()) throw ParseError("no objective row");
        const size_t m = md.row_names.size();
        row_data();
        column_bounds();
        md.row_lo.resize(m), md.row_up.resize(m);
        for (size_t i = 0; i < m; ++i) row_bounds(row_kind_[i], rhs_[i], has_range_[i] != 0, range_[i],
                                                  md.row_lo[i], md.row_up[i]);
        for (std::vector<double>* lower : {&md.col_lo, &md.row_lo})
            for (double& v : *lower)
                if (v <= -kHuge) md.sentinel_bounds += std::isfinite(v) ? 1 : 0, v = -kInf;
        for (std::vector<double>* upper : {&md.col_up, &md.row_up})
            for (double& v : *upper)
                if (v >= kHuge) md.sentinel_bounds += std::isfinite(v) ? 1 : 0, v = kInf;
        return std::move(md);
    }

  private:
    struct Entry {
        int32_t row;
        double v;
    };
    NameTable rows_, cols_;
    std::string objective_;
    std::unordered_set<std::string_view> ignored_rows_;
    std::vector<char> row_kind_;
    std::vector<double> rhs_, range_;
    std::vector<char> has_range_;
    bool in_integer_block_ = false;
    int current_ = -1;
    std::string_view current_name_;
    std::vector<Entry> pending_;
    std::map<std::pair<int, int>, double> quad_;

    static void row_bounds(char kind, double b, bool ranged, double r, double& lo, double& up) {
        switch (kind) {
            case 'E':
                lo = up = b;
                if (ranged) (r >= 0 ? up : lo) = b + r;
                break;
            case 'L':
                up = b, lo = ranged ? b - std::fabs(r) : -kInf;
                break;
            default:  // 'G'
                lo = b, up = ranged ? b + std::fabs(r) : kInf;
        }
    }
    // The current column's entries, by row (stable: one row's entries keep their file order), summed per row;
    // zero sums are dropped.
    void close_column() {
        if (current_ < 0) return;
        auto by_row = [](const Entry& a, const Entry& b) { return a.row < b.row; };
        if (pending_.size() <= 32) {  // insertion sort: no buffer per column
            for (size_t k = 1; k < pending_.size(); ++k)
                for (size_t w = k; w > 0 && by_row(pending_[w], pending_[w - 1]); --w) std::swap(pending_[w], pending_[w - 1]);
        } else {
            std::stable_sort(pending_.begin(), pending_.end(), by_row);
        }
        size_t k = 0;
        while (k < pending_.size()) {
            const int32_t r = pending_[k].row;
            double sum = 0;
            bool first = true;
            for (; k < pending_.size() && pending_[k].row == r; ++k) sum = first ? pending_[k].v : sum + pending_[k].v, first = false;
            if (sum != 0) md.row_idx.push_back(r), md.val.push_back(sum);
        }
        md.col_ptr.push_back(int64_t(md.row_idx.size()));
        pending_.clear();
    }
};

// ------------------------------------------------------------------------------------------------ parallel paths
// A COLUMNS record: an entry (column, row reference, value), or an integer marker (kind 1 opens, 2 closes).
struct ColumnRecord {
    std::string_view col;
    int row;
    int kind;
    double v;
};

void marker_line(const Fields& f, bool& opens) {
    bool open = false, close = false;
    for (std::string_view w : f) open |= w == "'INTORG'", close |= w == "'INTEND'";
    if (open == close) throw ParseError("bad MARKER line");
    opens = open;
}
bool is_marker(const Fields& f) { return f.size() >= 2 && f[1] == "'MARKER'"; }

// Tokenise free-format COLUMNS lines of buf[b, e) on `parts` threads (records per chunk, chunks in file order).
// False when any line is malformed: the section is then read line by line, which reports the first error.
bool tokenize_columns(const std::string& buf, size_t b, size_t e, int parts, const ModelBuilder& mb,
                      std::vector<std::vector<ColumnRecord>>& out) {
    const std::vector<size_t> cut = chunk_cuts(buf, b, e, parts);
    out.assign(size_t(parts), {});
    std::vector<char> failed(size_t(parts), 0);
    on_threads(parts, [&](int q) {
        Fields f;
        std::vector<ColumnRecord>& recs = out[size_t(q)];
        recs.reserve((cut[size_t(q) + 1] - cut[size_t(q)]) / 16 + 16);  // an entry takes at least 16 bytes of text
        LineCursor cur(buf, cut[size_t(q)], cut[size_t(q) + 1]);
        std::string_view line;
        try {
            while (cur.next(line)) {
                free_fields(line, f);
                if (is_marker(f)) {
                    bool opens = false;
                    marker_line(f, opens);
                    recs.push_back({std::string_view(), 0, opens ? 1 : 2, 0.0});
                    continue;
                }
                if (f.size() != 3 && f.size() != 5) throw ParseError("bad COLUMNS line");
                for (size_t k = 1; k + 1 < f.size(); k += 2) recs.push_back({f[0], mb.row(f[k]), 0, parse_number(f[k + 1])});
            }
        } catch (const ParseError&) {
            failed[size_t(q)] = 1;
        }
    });
    return std::find(failed.begin(), failed.end(), 1) == failed.end();
}

// A BOUNDS record: the set named on the line (may be empty), the column, the type and value, or the line's error.
// A malformed line's error (`early`) comes before the set test; the others after it, as line by line.
struct BoundRecord {
    std::string_view set, type;
    int col = -1, err = -1;  // err: index into the chunk's messages, -1 if none
    bool early = false;
    double v = 0;
};

// Free-format BOUNDS fields -> (set, column, value) by the field count and the type.
bool bound_fields(const Fields& f, std::string_view& set, std::string_view& col, std::string_view& val) {
    const bool no_value = !f.empty() && bound_has_no_value(f[0]);
    switch (f.size()) {
        case 4: set = f[1], col = f[2], val = f[3]; return true;
        case 3:
            if (no_value) set = f[1], col = f[2];
            else col = f[1], val = f[2];
            return true;
        case 2: col = f[1]; return true;
        default: return false;
    }
}

void tokenize_bounds(const std::string& buf, size_t b, size_t e, int parts, const ModelBuilder& mb,
                     std::vector<std::vector<BoundRecord>>& out, std::vector<std::vector<std::string>>& msgs) {
    const std::vector<size_t> cut = chunk_cuts(buf, b, e, parts);
    out.assign(size_t(parts), {});
    msgs.assign(size_t(parts), {});
    on_threads(parts, [&](int q) {
        Fields f;
        std::vector<BoundRecord>& recs = out[size_t(q)];
        std::vector<std::string>& msg = msgs[size_t(q)];
        recs.reserve((cut[size_t(q) + 1] - cut[size_t(q)]) / 12 + 16);
        LineCursor cur(buf, cut[size_t(q)], cut[size_t(q) + 1]);
        std::string_view line;
        while (cur.next(line)) {
            free_fields(line, f);
            BoundRecord r;
            auto fail = [&](std::string m, bool early) {
                r.err = int(msg.size()), r.early = early;
                msg.push_back(std::move(m));
            };
            r.type = f.empty() ? std::string_view() : f[0];
            std::string_view col, val;
            if (!bound_fields(f, r.set, col, val)) {
                fail("bad BOUNDS line", true);
            } else if (const int* j = mb.find_column(col); !j) {
                fail("unknown column '" + std::string(col) + "' in BOUNDS", false);
            } else {
                r.col = *j;
                try {
                    r.v = bound_has_no_value(r.type) || val.empty() ? 0 : parse_number(val);
                    if (bound_kind(r.type) == BoundKind::Invalid) fail("unsupported bound type " + std::string(r.type), false);
                } catch (const ParseError& ex) {
                    fail(ex.what(), false);
                }
            }
            recs.push_back(r);
        }
    });
}

// ------------------------------------------------------------------------------------------------ the reader
std::string read_file(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw ParseError("cannot open " + path);
    in.seekg(0, std::ios::end);
    const std::streamoff size = in.tellg();
    in.seekg(0, std::ios::beg);
    std::string buf(size > 0 ? size_t(size) : 0, '\0');
    if (size > 0 && !in.read(&buf[0], size)) throw ParseError("cannot read " + path);
    return buf;
}

class Reader {
  public:
    Reader(const std::string& buf, bool fixed) : buf_(buf), fixed_(fixed), mb_(buf.size()) {}

    Model read() {
        LineCursor cur(buf_, 0, buf_.size());
        std::string_view line;
        bool ended = false;
        while (cur.next(line)) {
            if (!is_header_line(line)) {
                data_line(line);
                continue;
            }
            if (header(line)) {
                ended = true;
                break;
            }
            if (!fixed_ && (sec_ == Section::Columns || sec_ == Section::Bounds)) bulk_section(cur);
        }
        if (!ended) throw ParseError("missing ENDATA");
        return mb_.finish();
    }

  private:
    const std::string& buf_;
    bool fixed_;
    ModelBuilder mb_;
    Section sec_ = Section::None;
    std::unordered_set<std::string> seen_;  // ROWS and COLUMNS appear once
    Fields f_;

    static void check_sense(ModelBuilder& mb, std::string_view w) {
        if (w == "MAX" || w == "MAXIMIZE") mb.md.maximize = true;
        else if (w != "MIN" && w != "MINIMIZE") throw ParseError("bad OBJSENSE " + std::string(w));
    }

    // A header line; returns true at ENDATA.
    bool header(std::string_view line) {
        Fields w;
        free_fields(line, w);
        const std::string name(w.empty() ? std::string_view() : w[0]);
        const std::string_view arg = w.size() > 1 ? w[1] : std::string_view();
        if (name == "ENDATA") return true;
        if (name == "NAME") {
            mb_.md.name = std::string(arg);
            sec_ = Section::None;
        } else if (name == "OBJSENSE") {
            if (!arg.empty()) check_sense(mb_, arg);
            sec_ = Section::ObjSense;
        } else if (name == "QUADOBJ" || name == "QMATRIX") {
            mb_.quad_full = name == "QMATRIX";
            sec_ = Section::Quad;
        } else if (name == "QSECTION" || name == "QCMATRIX") {
            if (name == "QCMATRIX" || arg != mb_.objective())
                throw ParseError("quadratic constraints are not supported (" + name + " " + std::string(arg) + ")");
            mb_.quad_full = true;
            sec_ = Section::Quad;
        } else if (name == "ROWS") {
            sec_ = Section::Rows;
        } else if (name == "COLUMNS") {
            sec_ = Section::Columns;
        } else if (name == "RHS") {
            sec_ = Section::Rhs;
        } else if (name == "RANGES") {
            sec_ = Section::Ranges;
        } else if (name == "BOUNDS") {
            sec_ = Section::Bounds;
        } else {
            throw ParseError("unsupported section " + name);
        }
        if ((sec_ == Section::Rows || sec_ == Section::Columns) && !seen_.insert(name).second)
            throw ParseError("section " + name + " appears twice");
        return false;
    }

    void data_line(std::string_view line) {
        if (fixed_) fixed_fields(line, sec_, f_);
        else free_fields(line, f_);
        const Fields& f = f_;
        switch (sec_) {
            case Section::None: break;
            case Section::ObjSense: check_sense(mb_, f.empty() ? std::string_view() : f[0]); break;
            case Section::Rows:
                if (f.size() != 2 || f[1].empty()) throw ParseError("bad ROWS line");
                mb_.declare_row(f[0], f[1]);
                break;
            case Section::Columns: columns_line(f); break;
            case Section::Rhs:
            case Section::Ranges: rhs_line(f, sec_ == Section::Rhs); break;
            case Section::Bounds: bounds_line(f); break;
            case Section::Quad: {
                if (f.size() != 3) throw ParseError("bad quadratic objective line");
                const int a = mb_.column(f[0]), b = mb_.column(f[1]);
                mb_.quad_term(a, b, parse_number(f[2]));
                break;
            }
        }
    }

    void columns_line(const Fields& f) {
        if (is_marker(f)) {
            bool opens = false;
            marker_line(f, opens);
            mb_.integer_marker(opens);
            return;
        }
        if (f.size() != 3 && f.size() != 5) throw ParseError("bad COLUMNS line");
        mb_.use_column(f[0]);
        for (size_t k = 1; k + 1 < f.size(); k += 2) {
            const int r = mb_.row(f[k]);
            mb_.add_entry(r, parse_number(f[k + 1]));
        }
    }

    // [set] row value [row value]: a set name leads the line in fixed format always, in free format when the
    // field count is odd
    void rhs_line(const Fields& f, bool rhs) {
        const size_t first = fixed_ || f.size() % 2 == 1 ? 1 : 0;
        if (first == 1 && !f[0].empty() && !ModelBuilder::in_first_set(rhs ? mb_.rhs_set : mb_.range_set, f[0])) return;
        mb_.row_data();
        for (size_t k = first; k + 1 < f.size(); k += 2) {
            const int r = mb_.row(f[k]);
            const double v = parse_number(f[k + 1]);
            if (rhs) mb_.set_rhs(r, v);
            else mb_.set_range(r, v);
        }
    }

    void bounds_line(const Fields& f) {
        mb_.column_bounds();
        const std::string_view type = f.empty() ? std::string_view() : f[0];
        std::string_view set, col, val;
        if (fixed_) {
            set = f.size() > 1 ? f[1] : std::string_view();
            col = f.size() > 2 ? f[2] : std::string_view();
            val = f.size() > 3 ? f[3] : std::string_view();
        } else if (!bound_fields(f, set, col, val)) {
            throw ParseError("bad BOUNDS line");
        }
        if (!set.empty() && !ModelBuilder::in_first_set(mb_.bound_set, set)) return;
        const int* j = mb_.find_column(col);
        if (!j) throw ParseError("unknown column '" + std::string(col) + "' in BOUNDS");
        mb_.apply_bound(*j, type, bound_has_no_value(type) || val.empty() ? 0 : parse_number(val));
    }

    // A COLUMNS or BOUNDS section of at least 2 MB in free format: tokenised on the host threads and applied in
    // file order (COLUMNS with a malformed line is left to the line-by-line pass, which reports its first error).
    void bulk_section(LineCursor& cur) {
        const size_t b = cur.pos(), e = section_end(buf_, b);
        const int parts = int(std::max<size_t>(1, std::min<size_t>(size_t(host_threads()), (e - b) >> 20)));
        if (parts < 2) return;
        if (sec_ == Section::Columns) {
            std::vector<std::vector<ColumnRecord>> recs;
            if (!tokenize_columns(buf_, b, e, parts, mb_, recs)) return;
            size_t entries = 0, starts = 0;  // capacity: entries, and an upper bound on the new columns
            for (const auto& part : recs) {
                entries += part.size();
                std::string_view prev;
                for (const ColumnRecord& c : part)
                    if (!c.kind && c.col != prev) ++starts, prev = c.col;
            }
            mb_.reserve_entries(entries, starts);
            for (const auto& part : recs)
                for (const ColumnRecord& c : part) {
                    if (c.kind) {
                        mb_.integer_marker(c.kind == 1);
                        continue;
                    }
                    mb_.use_column(c.col);
                    mb_.add_entry(c.row, c.v);
                }
        } else {
            std::vector<std::vector<BoundRecord>> recs;
            std::vector<std::vector<std::string>> msgs;
            tokenize_bounds(buf_, b, e, parts, mb_, recs, msgs);
            mb_.column_bounds();
            for (size_t q = 0; q < recs.size(); ++q)
                for (const BoundRecord& r : recs[q]) {
                    if (r.err >= 0 && r.early) throw ParseError(msgs[q][size_t(r.err)]);
                    if (!r.set.empty() && !ModelBuilder::in_first_set(mb_.bound_set, r.set)) continue;
                    if (r.err >= 0) throw ParseError(msgs[q][size_t(r.err)]);
                    mb_.apply_bound(r.col, r.type, r.v);
                }
        }
        cur.seek(e);
    }
};

Model parse(const std::string& buf, bool fixed) { return Reader(buf, fixed).read(); }

}  // namespace

// Free format first; a file that fails there is read in fixed columns. When both fail, the error names both unless
// they agree.
Model read_mps(const std::string& path) {
    const std::string buf = read_file(path);
    try {
        return parse(buf, false);
    } catch (const ParseError& free_err) {
        try {
            return parse(buf, true);
        } catch (const ParseError& fixed_err) {
            if (std::string(free_err.what()) == fixed_err.what()) throw;
            throw ParseError(std::string(free_err.what()) + " (free format); " + fixed_err.what() + " (fixed columns)");
        }
    }
}

taral_model Model::view() const {
    taral_model v{};
    v.m = int(row_lo.size()), v.n = int(cost.size());
    v.col_ptr = col_ptr.data(), v.row_idx = row_idx.data(), v.val = val.data();
    v.cost = cost.data(), v.col_lo = col_lo.data(), v.col_up = col_up.data();
    v.row_lo = row_lo.data(), v.row_up = row_up.data();
    v.obj_const = obj_const, v.maximize = maximize ? 1 : 0;
    v.is_int = is_int.data(), v.n_quadratic = n_quadratic;
    return v;
}

}  // namespace taral
