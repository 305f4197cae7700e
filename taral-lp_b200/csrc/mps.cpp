// MPS reader with the semantics of the reference reader (src/mps.cpp:1-399): whitespace-separated fields first,
// fixed columns as the fallback; OBJSENSE, RANGES, the usual bound types, integer MARKER blocks and quadratic
// objective sections; only the first named RHS / RANGES / BOUNDS set is used. Malformed input is an error:
// missing ENDATA, a repeated ROWS or COLUMNS section, duplicate row names, a column in two separate blocks,
// names used before they are declared and numbers outside the plain decimal grammar (hex, inf, nan, overflow).
// Entries of one column are sorted by row, duplicates summed in file order and zero sums dropped.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <charconv>
#include <string_view>
#include <thread>
#include <unordered_map>
#include <unordered_set>

#include "host.hpp"

namespace taral {
namespace {

constexpr double kHuge = 1e20;  // |bound| >= 1e20 is infinite

double parse_number(std::string_view s) {
    size_t i = 0, n = s.size();
    auto digits = [&] {
        size_t a = i;
        while (i < n && std::isdigit(static_cast<unsigned char>(s[i]))) ++i;
        return i - a;
    };
    if (i < n && (s[i] == '+' || s[i] == '-')) ++i;
    size_t mant = digits();
    if (i < n && s[i] == '.') ++i, mant += digits();
    bool ok = mant > 0;
    if (ok && i < n && std::strchr("eEdD", s[i])) {
        ++i;
        if (i < n && (s[i] == '+' || s[i] == '-')) ++i;
        ok = digits() > 0;
    }
    if (!ok || i != n) throw ParseError("bad number '" + std::string(s) + "'");
    char small[96];
    std::string big;
    char* t = small;
    if (n + 1 > sizeof small) big.resize(n + 1), t = &big[0];
    for (size_t k = 0; k < n; ++k) t[k] = (s[k] == 'd' || s[k] == 'D') ? 'E' : s[k];
    t[n] = 0;
    // from_chars rounds correctly like strtod (the same double); out-of-range text goes to strtod, whose overflow /
    // underflow results the checks below and the callers expect
    double v = 0;
    const auto r = std::from_chars(t, t + n, v);
    if (r.ec != std::errc() || r.ptr != t + n) v = std::strtod(t, nullptr);
    if (!std::isfinite(v)) throw ParseError("number '" + std::string(s) + "' is not finite");
    return v;
}

std::string_view fixed_field(std::string_view line, size_t a, size_t b) {
    if (line.size() <= a) return {};
    std::string_view s = line.substr(a, b - a);
    size_t i = s.find_first_not_of(" \t"), j = s.find_last_not_of(" \t\r");
    return i == std::string_view::npos ? std::string_view() : s.substr(i, j - i + 1);
}

// Tokens of one data line (views into the line): whitespace-separated (free format) or the fixed-column fields.
void split(std::string_view line, const std::string& section, bool fixed, std::vector<std::string_view>& t) {
    t.clear();
    if (!fixed) {
        auto ws = [](char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; };
        size_t p = 0, e = line.size();
        while (p < e) {
            while (p < e && ws(line[p])) ++p;
            size_t s = p;
            while (p < e && !ws(line[p])) ++p;
            if (p > s) t.push_back(line.substr(s, p - s));
        }
        return;
    }
    auto f = [&](size_t a, size_t b) { t.push_back(fixed_field(line, a, b)); };
    if (section == "ROWS") {
        f(1, 3), f(4, 12);
    } else if (section == "BOUNDS") {
        f(1, 3), f(4, 12), f(14, 22);
        if (!fixed_field(line, 24, 36).empty()) f(24, 36);
    } else {
        f(4, 12), f(14, 22), f(24, 36);
        if (!fixed_field(line, 39, 47).empty()) f(39, 47), f(49, 61);
    }
}

struct Entry {
    int32_t row;
    double v;
};

// Name -> index for the ROWS and COLUMNS names: open addressing with linear probing, grown at half load. A slot
// is 8 bytes (the upper half of a 64-bit FNV-1a hash and the index), so a probe costs one cache line; a tag match
// is confirmed against the name of that index, a view into the file buffer (the buffer outlives the table).
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
    bool count(std::string_view k) const { return find(k) != nullptr; }
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
    int add(std::string_view k) {  // k must not be present; indices are 0, 1, 2, ... in insertion order
        if (2 * (name_.size() + 1) > slot_.size()) rehash(2 * slot_.size());
        const int v = int(name_.size());
        name_.push_back(k);
        place(hash(k), v);
        return v;
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

// One entry of the COLUMNS section, tokenised: an entry (col, row as row_of gives it, value) or a MARKER line
// (kind 1: INTORG, 2: INTEND).
struct ColRec {
    std::string_view col;
    int row;
    int kind;
    double v;
};

bool is_header(std::string_view line) {  // a section header: not blank, not a comment, not indented
    return line.find_first_not_of(" \t") != std::string_view::npos && line[0] != ' ' && line[0] != '\t' &&
           line[0] != '*';
}

// Tokenise the free-format COLUMNS lines in [b, e) of buf on `threads` threads (line-aligned chunks, one record
// list each; read in chunk order they are in file order). Returns false if any line is malformed: the caller then
// parses sequentially, which reports the same first error as always.
template <class RowOf>
bool tokenize_columns(const std::string& buf, size_t b, size_t e, int threads, const RowOf& row_of,
                      std::vector<std::vector<ColRec>>& parts) {
    std::vector<size_t> cut{b};
    for (int q = 1; q < threads; ++q) {
        size_t p = b + (e - b) * size_t(q) / size_t(threads);
        p = std::max(p, cut.back());
        const size_t nl = buf.find('\n', p);
        cut.push_back(nl == std::string::npos || nl >= e ? e : nl + 1);
    }
    cut.push_back(e);
    const size_t nparts = static_cast<size_t>(threads);
    parts.assign(nparts, std::vector<ColRec>());
    std::vector<char> bad(nparts, 0);
    auto work = [&](int q) {
        std::vector<std::string_view> t;
        std::vector<ColRec>& r = parts[size_t(q)];
        r.reserve((cut[size_t(q) + 1] - cut[size_t(q)]) / 16 + 16);  // an entry takes at least 16 bytes of text
        try {
            for (size_t pos = cut[size_t(q)]; pos < cut[size_t(q) + 1];) {
                size_t nl = buf.find('\n', pos);
                if (nl == std::string::npos || nl > cut[size_t(q) + 1]) nl = cut[size_t(q) + 1];
                std::string_view line(buf.data() + pos, nl - pos);
                pos = nl + 1;
                if (!line.empty() && line.back() == '\r') line.remove_suffix(1);
                if (line.find_first_not_of(" \t") == std::string_view::npos || line[0] == '*') continue;
                split(line, "COLUMNS", false, t);
                if (t.size() >= 2 && t[1] == "'MARKER'") {
                    bool st = false, en = false;
                    for (std::string_view w : t) st |= w == "'INTORG'", en |= w == "'INTEND'";
                    if (st == en) throw ParseError("bad MARKER line");
                    r.push_back({std::string_view(), 0, st ? 1 : 2, 0.0});
                    continue;
                }
                if (t.size() != 3 && t.size() != 5) throw ParseError("bad COLUMNS line");
                for (size_t k = 1; k + 1 < t.size(); k += 2) r.push_back({t[0], row_of(t[k]), 0, parse_number(t[k + 1])});
            }
        } catch (const ParseError&) {
            bad[size_t(q)] = 1;
        }
    };
    std::vector<std::thread> pool;
    for (int q = 1; q < threads; ++q) pool.emplace_back(work, q);
    work(0);
    for (auto& th : pool) th.join();
    for (char x : bad)
        if (x) return false;
    return true;
}

// The offset where the section starting at pos ends: the next section header line, or the end of the buffer.
size_t section_end(const std::string& buf, size_t pos) {
    size_t end = pos;
    while (end < buf.size()) {
        size_t nl = buf.find('\n', end);
        if (nl == std::string::npos) nl = buf.size();
        std::string_view l(buf.data() + end, nl - end);
        if (!l.empty() && l.back() == '\r') l.remove_suffix(1);
        if (is_header(l)) break;
        end = nl + 1;
    }
    return std::min(end, buf.size());
}

// One line of the BOUNDS section, tokenised: the bound set named on the line (may be empty), the column, the
// bound type (index into kBoundTypes) and value, or the line's error: `early` errors (a malformed line) come before
// the bound-set test, the others (unknown column, bad number, unsupported type) after it, as in the sequential pass.
constexpr std::string_view kBoundTypes[] = {"LO", "UP", "FX", "FR", "MI", "PL", "BV", "LI", "UI"};
struct BoundRec {
    std::string_view set;
    int col = -1, type = -1, err = -1;  // err: index into the chunk's messages, -1 if none
    bool early = false;
    double v = 0;
};

// Tokenise the free-format BOUNDS lines in [b, e) of buf on `threads` threads (line-aligned chunks, records and
// error messages per chunk, in file order). Column names are looked up in col_of (read only).
template <class ColOf>
void tokenize_bounds(const std::string& buf, size_t b, size_t e, int threads, const ColOf& col_of,
                     std::vector<std::vector<BoundRec>>& parts, std::vector<std::vector<std::string>>& errs) {
    std::vector<size_t> cut{b};
    for (int q = 1; q < threads; ++q) {
        size_t p = std::max(b + (e - b) * size_t(q) / size_t(threads), cut.back());
        const size_t nl = buf.find('\n', p);
        cut.push_back(nl == std::string::npos || nl >= e ? e : nl + 1);
    }
    cut.push_back(e);
    const size_t nparts = static_cast<size_t>(threads);
    parts.assign(nparts, std::vector<BoundRec>());
    errs.assign(nparts, std::vector<std::string>());
    auto work = [&](int q) {
        std::vector<std::string_view> t;
        std::vector<BoundRec>& out = parts[size_t(q)];
        std::vector<std::string>& msg = errs[size_t(q)];
        out.reserve((cut[size_t(q) + 1] - cut[size_t(q)]) / 12 + 16);
        for (size_t pos = cut[size_t(q)]; pos < cut[size_t(q) + 1];) {
            size_t nl = buf.find('\n', pos);
            if (nl == std::string::npos || nl > cut[size_t(q) + 1]) nl = cut[size_t(q) + 1];
            std::string_view line(buf.data() + pos, nl - pos);
            pos = nl + 1;
            if (!line.empty() && line.back() == '\r') line.remove_suffix(1);
            if (line.find_first_not_of(" \t") == std::string_view::npos || line[0] == '*') continue;
            split(line, "BOUNDS", false, t);
            BoundRec r;
            auto fail = [&](std::string m, bool early) {
                r.err = int(msg.size()), r.early = early;
                msg.push_back(std::move(m));
            };
            const std::string_view type = t.empty() ? std::string_view() : t[0];
            const bool no_value = type == "FR" || type == "MI" || type == "PL" || type == "BV";
            std::string_view col, val;
            if (t.size() == 4) {
                r.set = t[1], col = t[2], val = t[3];
            } else if (t.size() == 3) {
                if (no_value) r.set = t[1], col = t[2];
                else col = t[1], val = t[2];
            } else if (t.size() == 2) {
                col = t[1];
            } else {
                fail("bad BOUNDS line", true);
            }
            if (r.err < 0) {
                const int* jc = col_of(col);
                if (!jc) {
                    fail("unknown column '" + std::string(col) + "' in BOUNDS", false);
                } else {
                    r.col = *jc;
                    try {
                        r.v = no_value || val.empty() ? 0 : parse_number(val);
                        for (int k = 0; k < 9; ++k)
                            if (type == kBoundTypes[k]) r.type = k;
                        if (r.type < 0) fail("unsupported bound type " + std::string(type), false);
                    } catch (const ParseError& ex) {
                        fail(ex.what(), false);
                    }
                }
            }
            out.push_back(r);
        }
    };
    std::vector<std::thread> pool;
    for (int q = 1; q < threads; ++q) pool.emplace_back(work, q);
    work(0);
    for (auto& th : pool) th.join();
}

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

// Row / column names are views into the file buffer, which outlives the parse.
Model parse(const std::string& path, bool fixed) {
    const std::string buf = read_file(path);
    Model md;
    std::string section, obj_row;
    NameTable row_id(buf.size() / 512 + 16), col_id(buf.size() / 256 + 16);
    std::unordered_set<std::string_view> free_rows;
    std::unordered_set<std::string> seen;
    std::vector<char> row_type;
    std::vector<double> rhs, range;
    std::vector<char> has_range;
    bool in_int = false, endata = false, q_full = false;
    int cur = -1;
    std::string_view cur_name;
    std::vector<Entry> pending;
    std::string rhs_set, range_set, bound_set;
    std::map<std::pair<int, int>, double> q;
    std::vector<std::string_view> t;

    auto close_column = [&] {  // sorted by row, duplicates summed in file order, zero sums dropped
        if (cur < 0) return;
        if (pending.size() <= 32) {  // stable insertion sort: no buffer to allocate per column
            for (size_t k = 1; k < pending.size(); ++k) {
                const Entry e = pending[k];
                size_t w = k;
                for (; w > 0 && pending[w - 1].row > e.row; --w) pending[w] = pending[w - 1];
                pending[w] = e;
            }
        } else {
            std::stable_sort(pending.begin(), pending.end(),
                             [](const Entry& a, const Entry& b) { return a.row < b.row; });
        }
        size_t start = md.row_idx.size();
        for (const Entry& e : pending) {
            if (md.row_idx.size() > start && md.row_idx.back() == e.row) md.val.back() += e.v;
            else md.row_idx.push_back(e.row), md.val.push_back(e.v);
        }
        size_t w = start;
        for (size_t k = start; k < md.row_idx.size(); ++k)
            if (md.val[k] != 0) md.row_idx[w] = md.row_idx[k], md.val[w] = md.val[k], ++w;
        md.row_idx.resize(w), md.val.resize(w);
        md.col_ptr.push_back(int64_t(w));
        pending.clear();
    };
    auto first_set = [](std::string& keep, std::string_view nm) {
        if (keep.empty()) keep = std::string(nm);
        return keep == nm;
    };
    auto row_of = [&](std::string_view nm) -> int {
        if (const int* r = row_id.find(nm)) return *r;
        if (nm == obj_row) return -1;
        if (free_rows.count(nm)) return -2;
        throw ParseError("unknown row '" + std::string(nm) + "'");
    };
    auto apply_bound = [&](int j, std::string_view type, double v) {  // one BOUNDS entry, in file order
        double &lo = md.col_lo[size_t(j)], &up = md.col_up[size_t(j)];
        if (type == "BV" || type == "LI" || type == "UI") md.is_int[size_t(j)] = 1;
        if (type == "LO" || type == "LI") lo = v;
        else if (type == "UP" || type == "UI") {
            up = v;
            if (v < 0 && lo == 0) lo = -kInf;
        } else if (type == "FX") lo = up = v;
        else if (type == "FR") lo = -kInf, up = kInf;
        else if (type == "MI") lo = -kInf;
        else if (type == "PL") up = kInf;
        else if (type == "BV") lo = 0, up = 1;
        else throw ParseError("unsupported bound type " + std::string(type));
    };
    auto col_of = [&](std::string_view nm) {
        const int* c = col_id.find(nm);
        if (!c) throw ParseError("unknown column '" + std::string(nm) + "'");
        return *c;
    };

    for (size_t pos = 0; pos < buf.size();) {
        size_t nl = buf.find('\n', pos);
        if (nl == std::string::npos) nl = buf.size();
        std::string_view line(buf.data() + pos, nl - pos);
        pos = nl + 1;
        if (!line.empty() && line.back() == '\r') line.remove_suffix(1);
        if (line.find_first_not_of(" \t") == std::string_view::npos || line[0] == '*') continue;
        if (line[0] != ' ' && line[0] != '\t') {  // section header
            std::istringstream hs{std::string(line)};
            std::string arg;
            hs >> section >> arg;
            if (section == "NAME") {
                md.name = arg;
            } else if (section == "ENDATA") {
                endata = true;
                break;
            } else if (section == "OBJSENSE") {
                if (!arg.empty()) {
                    if (arg == "MAX" || arg == "MAXIMIZE") md.maximize = true;
                    else if (arg != "MIN" && arg != "MINIMIZE") throw ParseError("bad OBJSENSE " + arg);
                }
            } else if (section == "QUADOBJ" || section == "QMATRIX") {
                q_full = section == "QMATRIX";
                section = "QUAD";
            } else if (section == "QSECTION" || section == "QCMATRIX") {
                if (section == "QCMATRIX" || arg != obj_row)
                    throw ParseError("quadratic constraints are not supported (" + section + " " + arg + ")");
                q_full = true;
                section = "QUAD";
            } else if (section != "ROWS" && section != "COLUMNS" && section != "RHS" && section != "RANGES" &&
                       section != "BOUNDS") {
                throw ParseError("unsupported section " + section);
            }
            if ((section == "ROWS" || section == "COLUMNS") && !seen.insert(section).second)
                throw ParseError("section " + section + " appears twice");
            if (section == "COLUMNS" && !fixed) {  // the bulk of a file: tokenised in parallel, merged in order
                const size_t end = section_end(buf, pos);
                std::vector<std::vector<ColRec>> parts;
                const int nt = int(std::max<size_t>(1, std::min<size_t>(size_t(host_threads()), (end - pos) >> 20)));
                if (nt > 1 && tokenize_columns(buf, pos, end, nt, row_of, parts)) {
                    size_t recs = 0, starts = 0;  // capacity: entries, and an upper bound on the new columns
                    for (const std::vector<ColRec>& part : parts) {
                        recs += part.size();
                        std::string_view prev;
                        for (const ColRec& c : part)
                            if (!c.kind && c.col != prev) ++starts, prev = c.col;
                    }
                    md.row_idx.reserve(md.row_idx.size() + recs), md.val.reserve(md.val.size() + recs);
                    md.col_names.reserve(md.col_names.size() + starts), md.cost.reserve(md.cost.size() + starts);
                    md.is_int.reserve(md.is_int.size() + starts), md.col_ptr.reserve(md.col_ptr.size() + starts);
                    for (const std::vector<ColRec>& part : parts)
                    for (const ColRec& c : part) {
                        if (c.kind) {
                            in_int = c.kind == 1;
                            continue;
                        }
                        int j;
                        if (cur >= 0 && c.col == cur_name) {
                            j = cur;
                        } else {
                            if (col_id.add_if_absent(c.col) >= 0)
                                throw ParseError("column '" + std::string(c.col) + "' is listed in two separate blocks");
                            close_column();
                            j = int(md.col_names.size());
                            md.col_names.emplace_back(c.col);
                            cur_name = c.col;
                            md.cost.push_back(0);
                            md.is_int.push_back(in_int ? 1 : 0);
                        }
                        cur = j;
                        if (c.row == -1) md.cost[j] += c.v;
                        else if (c.row >= 0) pending.push_back({c.row, c.v});
                    }
                    pos = end;
                }
            }
            if (section == "BOUNDS" && !fixed) {  // one line per bounded column: tokenised in parallel as well
                const size_t end = section_end(buf, pos);
                const int nt = int(std::max<size_t>(1, std::min<size_t>(size_t(host_threads()), (end - pos) >> 20)));
                if (nt > 1) {
                    std::vector<std::vector<BoundRec>> parts;
                    std::vector<std::vector<std::string>> errs;
                    tokenize_bounds(buf, pos, end, nt, [&](std::string_view nm) { return col_id.find(nm); }, parts,
                                    errs);
                    if (md.col_lo.empty()) {
                        md.col_lo.assign(md.col_names.size(), 0);
                        md.col_up.assign(md.col_names.size(), kInf);
                    }
                    for (size_t q = 0; q < parts.size(); ++q)
                        for (const BoundRec& r : parts[q]) {
                            if (r.err >= 0 && r.early) throw ParseError(errs[q][size_t(r.err)]);
                            if (!r.set.empty() && !first_set(bound_set, r.set)) continue;
                            if (r.err >= 0) throw ParseError(errs[q][size_t(r.err)]);
                            apply_bound(r.col, kBoundTypes[r.type], r.v);
                        }
                    pos = end;
                }
            }
            continue;
        }
        split(line, section, fixed, t);
        if (section == "OBJSENSE") {
            std::string_view v = t.empty() ? std::string_view() : t[0];
            if (v == "MAX" || v == "MAXIMIZE") md.maximize = true;
            else if (v != "MIN" && v != "MINIMIZE") throw ParseError("bad OBJSENSE " + std::string(v));
        } else if (section == "ROWS") {
            if (t.size() != 2 || t[1].empty()) throw ParseError("bad ROWS line");
            char type = t[0].empty() ? '?' : char(std::toupper(static_cast<unsigned char>(t[0][0])));
            if (row_id.count(t[1]) || t[1] == obj_row || free_rows.count(t[1]))
                throw ParseError("duplicate row name '" + std::string(t[1]) + "'");
            if (type == 'N') {
                if (obj_row.empty()) obj_row = std::string(t[1]);
                else free_rows.insert(t[1]);
            } else if (type == 'E' || type == 'L' || type == 'G') {
                row_id.add(t[1]);
                md.row_names.emplace_back(t[1]);
                row_type.push_back(type);
            } else {
                throw ParseError("bad row type " + std::string(t[0]));
            }
        } else if (section == "COLUMNS") {
            if (t.size() >= 2 && t[1] == "'MARKER'") {
                bool s = false, e = false;
                for (std::string_view w : t) s |= w == "'INTORG'", e |= w == "'INTEND'";
                if (s == e) throw ParseError("bad MARKER line");
                in_int = s;
                continue;
            }
            if (t.size() != 3 && t.size() != 5) throw ParseError("bad COLUMNS line");
            int j;
            if (cur >= 0 && t[0] == cur_name) {
                j = cur;
            } else {
                if (col_id.add_if_absent(t[0]) >= 0)
                    throw ParseError("column '" + std::string(t[0]) + "' is listed in two separate blocks");
                close_column();
                j = int(md.col_names.size());
                md.col_names.emplace_back(t[0]);
                cur_name = t[0];
                md.cost.push_back(0);
                md.is_int.push_back(in_int ? 1 : 0);
            }
            cur = j;
            for (size_t k = 1; k + 1 < t.size(); k += 2) {
                int r = row_of(t[k]);
                double v = parse_number(t[k + 1]);
                if (r == -1) md.cost[j] += v;
                else if (r >= 0) pending.push_back({r, v});
            }
        } else if (section == "RHS" || section == "RANGES") {
            size_t start = fixed ? 1 : (t.size() % 2 == 1 ? 1 : 0);
            if (start == 1 && !t[0].empty() && !first_set(section == "RHS" ? rhs_set : range_set, t[0])) continue;
            if (rhs.empty()) {
                rhs.assign(md.row_names.size(), 0);
                range.assign(md.row_names.size(), 0);
                has_range.assign(md.row_names.size(), 0);
            }
            for (size_t k = start; k + 1 < t.size(); k += 2) {
                int r = row_of(t[k]);
                double v = parse_number(t[k + 1]);
                if (section == "RHS") {
                    if (r == -1) md.obj_const = -v;
                    else if (r >= 0) rhs[r] = v;
                } else if (r >= 0) {
                    range[r] = v, has_range[r] = 1;
                }
            }
        } else if (section == "BOUNDS") {
            if (md.col_lo.empty()) {
                md.col_lo.assign(md.col_names.size(), 0);
                md.col_up.assign(md.col_names.size(), kInf);
            }
            std::string_view type = t.empty() ? std::string_view() : t[0];
            bool no_value = type == "FR" || type == "MI" || type == "PL" || type == "BV";
            std::string_view set, col, val;
            if (fixed) {
                set = t.size() > 1 ? t[1] : std::string_view(), col = t.size() > 2 ? t[2] : std::string_view();
                val = t.size() > 3 ? t[3] : std::string_view();
            } else if (t.size() == 4) {
                set = t[1], col = t[2], val = t[3];
            } else if (t.size() == 3) {
                if (no_value) set = t[1], col = t[2];
                else col = t[1], val = t[2];
            } else if (t.size() == 2) {
                col = t[1];
            } else {
                throw ParseError("bad BOUNDS line");
            }
            if (!set.empty() && !first_set(bound_set, set)) continue;
            const int* jc = col_id.find(col);
            if (!jc) throw ParseError("unknown column '" + std::string(col) + "' in BOUNDS");
            apply_bound(*jc, type, no_value || val.empty() ? 0 : parse_number(val));
        } else if (section == "QUAD") {
            if (t.size() != 3) throw ParseError("bad quadratic objective line");
            int a = col_of(t[0]), b = col_of(t[1]);
            double v = parse_number(t[2]);
            if (q_full && a < b) continue;
            q[{std::max(a, b), std::min(a, b)}] += v;
        }
    }
    close_column();
    if (!endata) throw ParseError("missing ENDATA");
    for (const auto& kv : q)
        if (kv.second != 0) ++md.n_quadratic;
    if (obj_row.empty()) throw ParseError("no objective row");

    size_t m = md.row_names.size(), n = md.col_names.size();
    if (md.col_ptr.size() != n + 1) throw ParseError("internal: column pointer size");
    if (rhs.empty()) rhs.assign(m, 0), range.assign(m, 0), has_range.assign(m, 0);
    if (md.col_lo.empty()) md.col_lo.assign(n, 0), md.col_up.assign(n, kInf);
    md.row_lo.resize(m), md.row_up.resize(m);
    for (size_t i = 0; i < m; ++i) {
        double b = rhs[i], R = range[i];
        double &lo = md.row_lo[i], &up = md.row_up[i];
        if (row_type[i] == 'E') {
            lo = up = b;
            if (has_range[i]) (R >= 0 ? up : lo) = b + R;
        } else if (row_type[i] == 'L') {
            up = b;
            lo = has_range[i] ? b - std::fabs(R) : -kInf;
        } else {
            lo = b;
            up = has_range[i] ? b + std::fabs(R) : kInf;
        }
    }
    for (std::vector<double>* lo : {&md.col_lo, &md.row_lo})
        for (double& v : *lo)
            if (v <= -kHuge) {
                if (std::isfinite(v)) ++md.sentinel_bounds;
                v = -kInf;
            }
    for (std::vector<double>* up : {&md.col_up, &md.row_up})
        for (double& v : *up)
            if (v >= kHuge) {
                if (std::isfinite(v)) ++md.sentinel_bounds;
                v = kInf;
            }
    return md;
}

}  // namespace

Model read_mps(const std::string& path) {
    try {
        return parse(path, false);
    } catch (const ParseError& free_err) {
        try {
            return parse(path, true);
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
