// mps.cpp -- MPS files in and out, at the speed of one pass over the bytes.
//
// The reference reader (src/mps/mps_reader.cpp) parses each line through a
// std::stringstream, resolves every term's row and column through
// std::string-keyed maps and accumulates each row in its own
// std::unordered_map. This reader loads the file in one read, splits lines and
// fields in place, resolves names through open-addressing tables of views into
// the buffer (with the current column cached, since COLUMNS records arrive
// grouped by column), collects coefficients as (row, column, value) triplets
// in file order and groups them at the end with a counting sort. Numbers take
// an exact fast path (a decimal with at most 19 significant digits whose
// significand is at most 2^53 and whose power of ten is at most 22 in
// magnitude is one correctly rounded IEEE multiplication or division of two
// exact doubles, Clinger 1990) and strtod otherwise, so every value is the
// double the reference reads.
//
// The sections, records, conventions, warnings and error messages restate the
// reference reader's (mps_reader.cpp:87-443, finalizeRowBounds :445-503,
// get_or_create_variable :505-527, add_coefficient :529-551, add_quadratic
// :553-580). pdlpgpu_mps_lp restates adapter::toCompiledLp
// (src/adapter/pdlp_adapter.cpp:21-189) and CompiledLp::validate
// (pdlp_engine/include/pdlp/compiled_lp.h:32-60).
#include "pdlpgpu.h"
#include "pdlpgpu_mps.h"

#include <algorithm>
#include <cerrno>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <string_view>
#include <thread>
#include <vector>

extern "C" void pdlpgpu_internal_set_error(const char* message);

struct pdlpgpu_mps {
    std::string name;
    int32_t sense = 0;   // 0 minimize, 1 maximize
    double offset = 0.0;
    std::vector<std::string> var_names, row_names, warnings;
    std::vector<int32_t> var_type;
    std::vector<double> var_lower, var_upper, row_lower, row_upper;
    std::vector<int32_t> obj_index;
    std::vector<double> obj_value;
    std::vector<int64_t> row_start;
    std::vector<int32_t> row_index;
    std::vector<double> row_value;
    std::vector<int32_t> q_i, q_j;
    std::vector<double> q_value;
    // The compiled LP of pdlpgpu_mps_lp (owned here).
    std::vector<int64_t> lp_start;
    std::vector<int32_t> lp_index;
    std::vector<double> lp_value, lp_objective;
};

namespace pdlpgpu {
namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();
enum : int32_t { kContinuous = 0, kInteger = 1, kBinary = 2 };   // model::VariableType
enum : char { kLess = 'L', kGreater = 'G', kEqual = 'E' };

using sv = std::string_view;

// The C locale's isspace, as operator>> splits fields, by table lookup.
struct SpaceTable {
    bool v[256] = {};
    SpaceTable() {
        for (unsigned char c : {' ', '\t', '\n', '\v', '\f', '\r'}) v[c] = true;
    }
};
const SpaceTable kSpace;
inline bool is_space(char c) { return kSpace.v[static_cast<unsigned char>(c)]; }

std::string upper(sv s) {
    std::string r(s);
    for (char& c : r) c = static_cast<char>(std::toupper(static_cast<unsigned char>(c)));
    return r;
}

// s, with its quotes removed, equals the upper-case `word` ignoring case
// (no allocation: this runs on every COLUMNS record).
bool keyword(sv s, sv word) {
    size_t k = 0;
    for (char c : s) {
        if (c == '\'' || c == '"') continue;
        if (k >= word.size() || std::toupper(static_cast<unsigned char>(c)) != word[k]) return false;
        ++k;
    }
    return k == word.size();
}

std::string unquoted(sv s) {
    std::string r;
    r.reserve(s.size());
    for (char c : s)
        if (c != '\'' && c != '"') r.push_back(c);
    return r;
}

// Open-addressing table from names (views into the file buffer) to dense
// indices 0, 1, 2, ... in insertion order. A slot is 16 bytes and holds names
// of up to 11 bytes inline, so resolving such a name touches one cache line;
// a longer name keeps a 32-bit tag of its hash in the slot and is compared
// with the stored view only when the tag matches. `hash` is exposed so a
// caller can prefetch a name's slot (`prefetch`) before it looks the name up
// (`find_hashed`).
class NameTable {
public:
    static constexpr size_t kInline = 11;

    NameTable() { rehash(1024); }

    int32_t size() const { return static_cast<int32_t>(names_.size()); }

    static uint64_t hash(sv s) {   // FNV-1a, then a final mix
        uint64_t h = 1469598103934665603ull;
        for (unsigned char c : s) h = (h ^ c) * 1099511628211ull;
        h ^= h >> 29;
        h *= 0xbf58476d1ce4e5b9ull;
        return h ^ (h >> 32);
    }

    void prefetch(uint64_t h) const { __builtin_prefetch(&slots_[h & mask_]); }

    int32_t find(sv key) const { return find_hashed(key, hash(key)); }

    int32_t find_hashed(sv key, uint64_t h) const {
        for (size_t p = h & mask_;; p = (p + 1) & mask_) {
            const Slot& s = slots_[p];
            if (s.index < 0) return -1;
            if (matches(s, key, h)) return s.index;
        }
    }

    // The key's index, inserting it (with the next index) when absent.
    int32_t insert(sv key) {
        if (2 * (names_.size() + 1) > slots_.size()) rehash(slots_.size() * 2);
        const uint64_t h = hash(key);
        for (size_t p = h & mask_;; p = (p + 1) & mask_) {
            Slot& s = slots_[p];
            if (s.index < 0) {
                fill(s, key, h, static_cast<int32_t>(names_.size()));
                names_.push_back(key);
                return s.index;
            }
            if (matches(s, key, h)) return s.index;
        }
    }

private:
    struct Slot {
        int32_t index;            // < 0: empty
        uint8_t len;              // inline length, or kLong
        char key[kInline];        // the name, or the hash tag for a long name
    };
    static_assert(sizeof(Slot) == 16, "16-byte slots");
    static constexpr uint8_t kLong = 255;

    static uint32_t tag_of(uint64_t h) { return static_cast<uint32_t>(h >> 32); }

    bool matches(const Slot& s, sv key, uint64_t h) const {
        if (key.size() <= kInline)
            return s.len == key.size() && std::memcmp(s.key, key.data(), key.size()) == 0;
        if (s.len != kLong) return false;
        uint32_t tag;
        std::memcpy(&tag, s.key, 4);
        return tag == tag_of(h) && names_[static_cast<size_t>(s.index)] == key;
    }

    static void fill(Slot& s, sv key, uint64_t h, int32_t index) {
        s.index = index;
        if (key.size() <= kInline) {
            s.len = static_cast<uint8_t>(key.size());
            std::memcpy(s.key, key.data(), key.size());
        } else {
            s.len = kLong;
            const uint32_t tag = tag_of(h);
            std::memcpy(s.key, &tag, 4);
        }
    }

    void rehash(size_t size) {
        std::vector<Slot> slots(size);
        for (Slot& s : slots) s.index = -1;
        const size_t mask = size - 1;
        for (size_t i = 0; i < names_.size(); ++i) {
            const uint64_t h = hash(names_[i]);
            size_t q = h & mask;
            while (slots[q].index >= 0) q = (q + 1) & mask;
            fill(slots[q], names_[i], h, static_cast<int32_t>(i));
        }
        slots_.swap(slots);
        mask_ = mask;
    }

    std::vector<Slot> slots_;
    std::vector<sv> names_;
    size_t mask_ = 0;
};

// Decimal syntax: [+-] (digits [. digits] | . digits) [(e|E) [+-] digits].
// Returns false when `s` is not of that form; otherwise sets `out` to the
// correctly rounded value, or returns false with `range` set when it
// overflows or underflows (strtod's ERANGE, which the reference refuses).
bool parse_decimal(sv s, double& out, bool& range) {
    range = false;
    size_t i = 0;
    const size_t n = s.size();
    bool neg = false;
    if (i < n && (s[i] == '+' || s[i] == '-')) neg = s[i++] == '-';
    uint64_t m = 0;
    int digits = 0;        // significant digits kept in m
    int dropped = 0;       // integer digits not kept (shift the exponent up)
    int frac = 0;          // fraction digits kept
    bool any = false, exact = true;
    for (; i < n && s[i] >= '0' && s[i] <= '9'; ++i) {
        any = true;
        if (m == 0 && s[i] == '0') continue;
        if (digits < 19) {
            m = m * 10 + static_cast<uint64_t>(s[i] - '0');
            ++digits;
        } else {
            exact = false;
            ++dropped;
        }
    }
    if (i < n && s[i] == '.') {
        ++i;
        for (; i < n && s[i] >= '0' && s[i] <= '9'; ++i) {
            any = true;
            if (m == 0 && s[i] == '0') {
                ++frac;
                continue;
            }
            if (digits < 19) {
                m = m * 10 + static_cast<uint64_t>(s[i] - '0');
                ++digits;
                ++frac;
            } else {
                exact = false;
            }
        }
    }
    if (!any) return false;
    long exp10 = 0;
    if (i < n && (s[i] == 'e' || s[i] == 'E')) {
        ++i;
        bool eneg = false;
        if (i < n && (s[i] == '+' || s[i] == '-')) eneg = s[i++] == '-';
        if (i >= n || s[i] < '0' || s[i] > '9') return false;
        for (; i < n && s[i] >= '0' && s[i] <= '9'; ++i)
            if (exp10 < 100000) exp10 = exp10 * 10 + (s[i] - '0');
        if (eneg) exp10 = -exp10;
    }
    if (i != n) return false;
    if (m == 0) {
        out = neg ? -0.0 : 0.0;
        return true;
    }
    const long e = exp10 + dropped - frac;
    static const double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,
                                      1e8,  1e9,  1e10, 1e11, 1e12, 1e13, 1e14, 1e15,
                                      1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};
    if (exact && m <= (uint64_t(1) << 53) && e >= -22 && e <= 22) {
        const double v = static_cast<double>(m);
        const double r = e >= 0 ? v * kPow10[e] : v / kPow10[-e];
        out = neg ? -r : r;
        return true;
    }
    // Everything else through std::from_chars (correctly rounded, as strtod;
    // it takes no leading '+'). A result that overflows, or underflows to a
    // subnormal or zero, is a range error, as strtod reports it.
    const char* b = s.data() + (s[0] == '+' ? 1 : 0);
    double r = 0.0;
    const auto res = std::from_chars(b, s.data() + n, r, std::chars_format::general);
    if (res.ec == std::errc::result_out_of_range ||
        (res.ec == std::errc() && (std::isinf(r) || std::fpclassify(r) == FP_SUBNORMAL || r == 0.0))) {
        range = true;
        return false;
    }
    if (res.ec != std::errc() || res.ptr != s.data() + n) return false;
    out = r;
    return true;
}

// A value read as `stream >> double` reads it in COLUMNS, BOUNDS and the
// quadratic sections: decimal syntax only.
bool parse_stream(sv s, double& out) {
    bool range = false;
    return parse_decimal(s, out, range);
}

// A value read as std::stod with full consumption (RHS, RANGES): strtod's
// wider syntax (inf, nan, hexadecimal) is accepted too; out of range is not.
bool parse_full(sv s, double& out) {
    bool range = false;
    if (parse_decimal(s, out, range)) return true;
    if (range || s.empty() || is_space(s[0])) return false;
    const std::string copy(s);
    errno = 0;
    char* end = nullptr;
    const double r = std::strtod(copy.c_str(), &end);
    if (errno == ERANGE || end != copy.c_str() + copy.size()) return false;
    out = r;
    return true;
}

struct ParseError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

[[noreturn]] void fail(const std::string& message, size_t line) {
    throw ParseError("MpsReader Error (line " + std::to_string(line) + "): " + message);
}

enum class Section { None, Name, ObjSense, Rows, Columns, Rhs, Ranges, Bounds, QuadObj, QMatrix, End };

class Reader {
public:
    explicit Reader(pdlpgpu_mps& out) : out_(out) {}

    void read(const std::string& path) {
        load(path);
        std::vector<sv> tok;
        size_t line_number = 0;
        const char* p = buf_.data();
        const char* const end = p + buf_.size();
        while (p < end) {
            const char* nl = static_cast<const char*>(std::memchr(p, '\n', static_cast<size_t>(end - p)));
            const char* le = nl ? nl : end;
            sv line(p, static_cast<size_t>(le - p));
            p = nl ? nl + 1 : end;
            ++line_number;
            if (!line.empty() && line.back() == '\r') line.remove_suffix(1);
            if (line.empty() || line[0] == '*') continue;
            split(line, tok);
            if (tok.empty()) continue;
            if (line[0] != ' ' && line[0] != '\t') {
                if (header(tok, line_number)) break;
                if (section_ == Section::Columns) p = columns_in_parallel(p, end, line_number);
                continue;
            }
            record(tok, line, line_number);
        }
        flush();
        finish();
    }

private:
    void load(const std::string& path) {
        FILE* f = std::fopen(path.c_str(), "rb");
        if (f == nullptr) throw ParseError("MpsReader Error: Unable to open file " + path);
        std::fseek(f, 0, SEEK_END);
        const long size = std::ftell(f);
        std::fseek(f, 0, SEEK_SET);
        buf_.resize(size > 0 ? static_cast<size_t>(size) : 0);
        const size_t got = buf_.empty() ? 0 : std::fread(&buf_[0], 1, buf_.size(), f);
        std::fclose(f);
        if (got != buf_.size()) throw ParseError("MpsReader Error: Unable to open file " + path);
    }

    static void split(sv line, std::vector<sv>& tok) {
        tok.clear();
        size_t i = 0;
        const size_t n = line.size();
        while (true) {
            while (i < n && is_space(line[i])) ++i;
            if (i >= n) break;
            const size_t b = i;
            while (i < n && !is_space(line[i])) ++i;
            tok.emplace_back(line.substr(b, i - b));
        }
    }

    void set_sense(sv t, size_t line) {
        const std::string s = upper(t);
        if (s == "MAX" || s == "MAXIMIZE") out_.sense = 1;
        else if (s == "MIN" || s == "MINIMIZE") out_.sense = 0;
        else fail("unknown OBJSENSE value '" + std::string(t) + "'", line);
    }

    // A section header; true at ENDATA.
    bool header(const std::vector<sv>& tok, size_t line) {
        flush();
        const std::string h = upper(tok[0]);
        if (h == "NAME") {
            section_ = Section::Name;
            if (tok.size() > 1) out_.name = std::string(tok[1]);
        } else if (h == "OBJSENSE" || h == "OBJSENS") {
            section_ = Section::ObjSense;
            if (tok.size() > 1) set_sense(tok[1], line);
        } else if (h == "ROWS") {
            section_ = Section::Rows;
        } else if (h == "COLUMNS") {
            section_ = Section::Columns;
        } else if (h == "RHS") {
            section_ = Section::Rhs;
        } else if (h == "RANGES") {
            section_ = Section::Ranges;
        } else if (h == "BOUNDS") {
            section_ = Section::Bounds;
        } else if (h == "QUADOBJ" || h == "QUADS") {
            section_ = Section::QuadObj;
        } else if (h == "QMATRIX" || h == "QUADOBJ2") {
            section_ = Section::QMatrix;
        } else if (h == "ENDATA") {
            section_ = Section::End;
            return true;
        } else if (h == "SOS") {
            fail("SOS constraints are not representable in model::Model; "
                 "parsing this file would silently drop them", line);
        } else if (h == "INDICATORS") {
            fail("indicator constraints are not representable in model::Model; "
                 "parsing this file would silently drop them", line);
        } else if (h == "QCMATRIX" || h == "QCROWS") {
            fail("quadratic constraints are not representable in "
                 "model::Model (Constraint carries only linearTerms)", line);
        } else {
            fail("unrecognised section header '" + std::string(tok[0]) + "'", line);
        }
        return false;
    }

    void warn(std::string message) { out_.warnings.push_back(std::move(message)); }
    // Warnings outside the FIFO's own resolution wait for it first.
    void warn_in_order(std::string message) {
        flush();
        warn(std::move(message));
    }

    bool is_free_row(sv name) const { return free_.find(name) >= 0; }

    int32_t column(sv name) {
        if (!last_col_name_.empty() && name == last_col_name_) return last_col_;
        const int32_t before = cols_.size();
        const int32_t j = cols_.insert(name);
        if (j == before) new_column(name, integer_marker_);
        last_col_name_ = name;
        last_col_ = j;
        return j;
    }

    // The variable's model entries, for a name just added to cols_.
    void new_column(sv name, bool integer) {
        out_.var_names.emplace_back(name);
        out_.var_type.push_back(integer ? kInteger : kContinuous);
        out_.var_lower.push_back(0.0);
        out_.var_upper.push_back(kInf);
        lower_explicit_.push_back(0);
        obj_sum_.push_back(0.0);
        obj_has_.push_back(0);
    }

    // ---- COLUMNS in parallel -------------------------------------------
    // A COLUMNS section of more than kParallelBytes is cut into chunks at
    // line boundaries, one per host thread. Its records only look rows up
    // (the rows are final once COLUMNS starts) and create columns, so each
    // thread resolves rows through the read-only tables and keeps its own
    // first-appearance list of columns it has not seen created, with the
    // integer-marker state its chunk has set so far (or "inherited"). The
    // merge, in chunk order, creates those columns in file order with their
    // types and appends terms, objective contributions and warnings in file
    // order: the model, the warnings and the first error are the sequential
    // reader's.
    static constexpr size_t kParallelBytes = size_t(8) << 20;

    struct ChunkWarn {
        int kind;   // 0: unknown row, 1: record without coefficients
        sv var, row;
    };
    struct Chunk {
        const char* begin = nullptr;
        const char* end = nullptr;
        std::vector<int32_t> t_row, t_col;   // t_col >= 0: existing column; < 0: ~(local index)
        std::vector<double> t_val;
        std::vector<int32_t> o_col;
        std::vector<double> o_val;
        std::vector<sv> new_cols;
        std::vector<int8_t> new_marker;      // -1: the state the chunk inherits
        std::vector<ChunkWarn> warns;
        int8_t end_marker = -1;
        size_t lines = 0;
        bool failed = false;
        size_t fail_line = 0;                // within the chunk, from 1
        std::string fail_message;
    };

    void parse_chunk(Chunk& c) const {
        NameTable local;
        std::vector<sv> tok;
        int8_t marker = -1;
        sv last_name;
        int32_t last_ref = 0;
        auto colref = [&](sv name) -> int32_t {
            if (!last_name.empty() && name == last_name) return last_ref;
            int32_t r = cols_.find(name);
            if (r < 0) {
                const int32_t before = local.size();
                const int32_t k = local.insert(name);
                if (k == before) {
                    c.new_cols.push_back(name);
                    c.new_marker.push_back(marker);
                }
                r = ~k;
            }
            last_name = name;
            last_ref = r;
            return r;
        };
        const char* p = c.begin;
        while (p < c.end) {
            const char* nl = static_cast<const char*>(std::memchr(p, '\n', static_cast<size_t>(c.end - p)));
            const char* le = nl ? nl : c.end;
            sv line(p, static_cast<size_t>(le - p));
            p = nl ? nl + 1 : c.end;
            ++c.lines;
            if (!line.empty() && line.back() == '\r') line.remove_suffix(1);
            if (line.empty() || line[0] == '*') continue;
            split(line, tok);
            if (tok.empty()) continue;
            if (tok.size() >= 3 && keyword(tok[1], "MARKER") &&
                (keyword(tok[2], "INTORG") || keyword(tok[2], "INTEND"))) {
                marker = keyword(tok[2], "INTORG") ? 1 : 0;
                c.end_marker = marker;
                last_name = sv();
                continue;
            }
            const sv var = tok[0];
            const int32_t col = colref(var);
            int pairs = 0;
            for (size_t k = 1; k < tok.size(); k += 2) {
                double value = 0.0;
                if (k + 1 >= tok.size() || !parse_stream(tok[k + 1], value)) {
                    c.failed = true;
                    c.fail_line = c.lines;
                    c.fail_message = "COLUMNS entry for '" + std::string(var) + "' row '" +
                                     std::string(tok[k]) + "' has no coefficient";
                    return;
                }
                ++pairs;
                const sv row = tok[k];
                if (row == objective_) {
                    c.o_col.push_back(col);
                    c.o_val.push_back(value);
                    continue;
                }
                const int32_t i = rows_.find(row);
                if (i >= 0) {
                    c.t_row.push_back(i);
                    c.t_col.push_back(col);
                    c.t_val.push_back(value);
                } else if (!is_free_row(row)) {
                    c.warns.push_back({0, var, row});
                }
            }
            if (pairs == 0) c.warns.push_back({1, var, sv()});
        }
    }

    // Parses the COLUMNS section starting at `p` in parallel when it is large;
    // returns where the sequential loop resumes (the next header, or `p`
    // unchanged for a small section).
    const char* columns_in_parallel(const char* p, const char* end, size_t& line_number) {
        unsigned threads = std::thread::hardware_concurrency();
        if (threads > 32) threads = 32;
        if (threads < 2) return p;
        // The section ends at the next header line.
        const char* q = p;
        while (q < end) {
            const char* nl = static_cast<const char*>(std::memchr(q, '\n', static_cast<size_t>(end - q)));
            const char* le = nl ? nl : end;
            sv line(q, static_cast<size_t>(le - q));
            if (!line.empty() && line.back() == '\r') line.remove_suffix(1);
            if (!line.empty() && line[0] != '*' && line[0] != ' ' && line[0] != '\t') {
                bool any = false;
                for (char ch : line) any = any || !is_space(ch);
                if (any) break;
            }
            q = nl ? nl + 1 : end;
        }
        const size_t bytes = static_cast<size_t>(q - p);
        if (bytes < kParallelBytes) return p;
        flush();
        std::vector<Chunk> chunks(threads);
        const char* b = p;
        for (unsigned k = 0; k < threads; ++k) {
            const char* e = k + 1 == threads ? q : p + bytes * (k + 1) / threads;
            if (e < b) e = b;
            if (k + 1 < threads && e < q) {
                const char* nl = static_cast<const char*>(std::memchr(e, '\n', static_cast<size_t>(q - e)));
                e = nl ? nl + 1 : q;
            }
            chunks[k].begin = b;
            chunks[k].end = e;
            b = e;
        }
        std::vector<std::thread> pool;
        for (unsigned k = 1; k < threads; ++k) pool.emplace_back([this, &chunks, k] { parse_chunk(chunks[k]); });
        parse_chunk(chunks[0]);
        for (std::thread& t : pool) t.join();
        // Merge in chunk order.
        bool marker = integer_marker_;
        size_t base = line_number;
        std::vector<int32_t> map;
        for (Chunk& c : chunks) {
            if (c.failed) fail(c.fail_message, base + c.fail_line);
            map.resize(c.new_cols.size());
            for (size_t k = 0; k < c.new_cols.size(); ++k) {
                const int32_t before = cols_.size();
                const int32_t j = cols_.insert(c.new_cols[k]);
                if (j == before) new_column(c.new_cols[k], c.new_marker[k] < 0 ? marker : c.new_marker[k] == 1);
                map[k] = j;
            }
            if (c.end_marker >= 0) marker = c.end_marker == 1;
            auto resolve = [&](int32_t r) { return r >= 0 ? r : map[static_cast<size_t>(~r)]; };
            for (size_t k = 0; k < c.o_col.size(); ++k) {
                const size_t j = static_cast<size_t>(resolve(c.o_col[k]));
                obj_sum_[j] += c.o_val[k];
                obj_has_[j] = 1;
            }
            for (int32_t& r : c.t_col) r = resolve(r);
            Segment sg;
            sg.row.swap(c.t_row);
            sg.col.swap(c.t_col);
            sg.val.swap(c.t_val);
            segs_.push_back(std::move(sg));
            for (const ChunkWarn& w : c.warns) {
                if (w.kind == 0)
                    warn("COLUMNS entry for '" + std::string(w.var) + "' names unknown row '" +
                         std::string(w.row) + "'; ignored");
                else
                    warn("COLUMNS record for '" + std::string(w.var) + "' carried no coefficients");
            }
            base += c.lines;
        }
        segs_.emplace_back();   // later sequential terms follow the chunks
        integer_marker_ = marker;
        last_col_name_ = sv();
        line_number = base;
        return q;
    }

    // A term on a constraint row waits in a short FIFO while its row's slot
    // is prefetched; terms are resolved in file order, and the FIFO is
    // flushed before any warning is issued and at every section change, so
    // the warnings come out in the reference's order.
    struct Pending {
        sv var, row;
        uint64_t hash;
        int32_t col;
        double value;
    };
    static constexpr int kAhead = 16;

    void coefficient(sv var, sv row, double value) {
        const int32_t j = column(var);
        if (row == objective_) {
            obj_sum_[static_cast<size_t>(j)] += value;
            obj_has_[static_cast<size_t>(j)] = 1;
            return;
        }
        const uint64_t h = NameTable::hash(row);
        rows_.prefetch(h);
        if (pending_count_ == kAhead) resolve_one();
        pending_[(pending_head_ + pending_count_) % kAhead] = Pending{var, row, h, j, value};
        ++pending_count_;
    }

    void resolve_one() {
        const Pending& p = pending_[pending_head_];
        pending_head_ = (pending_head_ + 1) % kAhead;
        --pending_count_;
        const int32_t i = rows_.find_hashed(p.row, p.hash);
        if (i >= 0) {
            Segment& sg = segs_.back();
            sg.row.push_back(i);
            sg.col.push_back(p.col);
            sg.val.push_back(p.value);
            return;
        }
        if (!is_free_row(p.row))
            warn("COLUMNS entry for '" + std::string(p.var) + "' names unknown row '" +
                 std::string(p.row) + "'; ignored");
    }

    void flush() {
        while (pending_count_ > 0) resolve_one();
    }

    void record(const std::vector<sv>& tok, sv line, size_t ln) {
        switch (section_) {
            case Section::ObjSense:
                set_sense(tok[0], ln);
                break;
            case Section::Rows: {
                const std::string s = upper(tok[0]);
                if (tok.size() < 2) fail("ROWS record missing a row name", ln);
                const sv name = tok[1];
                if (s == "N") {
                    if (objective_.empty()) {
                        objective_ = name;
                    } else {
                        free_.insert(name);
                        warn("free row '" + std::string(name) + "' after the objective row was ignored");
                    }
                    break;
                }
                if (s != "L" && s != "G" && s != "E")
                    fail("unknown row sense '" + std::string(tok[0]) + "' for row '" +
                         std::string(name) + "'", ln);
                if (rows_.find(name) >= 0) fail("duplicate row name '" + std::string(name) + "'", ln);
                rows_.insert(name);
                out_.row_names.emplace_back(name);
                sense_.push_back(s[0]);
                rhs_.push_back(0.0);
                range_.push_back(0.0);
                has_range_.push_back(0);
                break;
            }
            case Section::Columns: {
                if (tok.size() >= 3 && keyword(tok[1], "MARKER") &&
                    (keyword(tok[2], "INTORG") || keyword(tok[2], "INTEND"))) {
                    {
                        integer_marker_ = keyword(tok[2], "INTORG");
                        last_col_name_ = sv();   // the marker changes how new columns are typed
                        break;
                    }
                }
                const sv var = tok[0];
                column(var);
                int pairs = 0;
                for (size_t k = 1; k < tok.size(); k += 2) {
                    double value = 0.0;
                    if (k + 1 >= tok.size() || !parse_stream(tok[k + 1], value))
                        fail("COLUMNS entry for '" + std::string(var) + "' row '" + std::string(tok[k]) +
                             "' has no coefficient", ln);
                    coefficient(var, tok[k], value);
                    ++pairs;
                }
                if (pairs == 0)
                    warn_in_order("COLUMNS record for '" + std::string(var) + "' carried no coefficients");
                break;
            }
            case Section::Rhs:
            case Section::Ranges: {
                const bool rhs = section_ == Section::Rhs;
                const bool named = tok.size() % 2 == 1;
                const size_t start = named ? 1 : 0;
                sv& selected = rhs ? rhs_vector_ : ranges_vector_;
                if (named) {
                    if (selected.empty()) selected = tok[0];
                    if (tok[0] != selected) {
                        warn(std::string(rhs ? "RHS" : "RANGES") + " vector '" + std::string(tok[0]) +
                             "' ignored; using first vector '" + std::string(selected) + "'");
                        break;
                    }
                }
                int pairs = 0;
                for (size_t k = start; k + 1 < tok.size(); k += 2) {
                    const sv row = tok[k];
                    double value = 0.0;
                    if (!parse_full(tok[k + 1], value))
                        fail(std::string(rhs ? "RHS" : "RANGES") + " entry for row '" + std::string(row) +
                             "' has a non-numeric value '" + std::string(tok[k + 1]) + "'", ln);
                    ++pairs;
                    if (row == objective_) {
                        if (rhs) offset_ = -value;
                        else warn("RANGES entry on the objective row was ignored");
                        continue;
                    }
                    const int32_t i = rows_.find(row);
                    if (i < 0) {
                        if (!rhs) warn("RANGES entry names unknown row '" + std::string(row) + "'; ignored");
                        else if (!is_free_row(row))
                            warn("RHS entry names unknown row '" + std::string(row) + "'; ignored");
                        continue;
                    }
                    if (rhs) {
                        rhs_[static_cast<size_t>(i)] = value;
                    } else {
                        range_[static_cast<size_t>(i)] = value;
                        has_range_[static_cast<size_t>(i)] = 1;
                    }
                }
                if (rhs && pairs == 0) warn("RHS record carried no entries");
                break;
            }
            case Section::Bounds:
                bound(tok, ln);
                break;
            case Section::QuadObj:
            case Section::QMatrix: {
                const sv col1 = tok[0];
                for (size_t k = 1; k < tok.size(); k += 2) {
                    double value = 0.0;
                    if (k + 1 >= tok.size() || !parse_stream(tok[k + 1], value))
                        fail("quadratic entry for '" + std::string(col1) + "', '" + std::string(tok[k]) +
                             "' has no value", ln);
                    const int32_t i = column(col1);
                    const int32_t j = column(tok[k]);
                    const bool mirror = section_ == Section::QuadObj;
                    q_lo_.push_back(std::min(i, j));
                    q_hi_.push_back(std::max(i, j));
                    q_val_.push_back(i == j ? value * 0.5 : (mirror ? value : value * 0.5));
                }
                break;
            }
            default:
                break;
        }
        (void)line;
    }

    void bound(const std::vector<sv>& tok, size_t ln) {
        // The bound type without allocating for the common ones.
        static const char* const kTypes[] = {"UP", "LO", "FX", "FR", "MI", "PL", "BV", "LI", "UI"};
        std::string type;
        for (const char* t : kTypes)
            if (keyword(tok[0], t)) {
                type = t;
                break;
            }
        if (type.empty()) type = upper(unquoted(tok[0]));
        if (tok.size() < 2) fail("BOUNDS record missing the bound-set name", ln);
        if (tok.size() < 3) fail("BOUNDS record missing a column name", ln);
        const sv var = tok[2];
        const size_t j = static_cast<size_t>(column(var));
        const bool needs_value = type == "LO" || type == "UP" || type == "FX" || type == "LI" || type == "UI";
        double value = 0.0;
        if (needs_value && (tok.size() < 4 || !parse_stream(tok[3], value)))
            fail("bound type '" + type + "' on column '" + std::string(var) + "' requires a value", ln);
        if ((type == "LI" || type == "UI") && (!std::isfinite(value) || std::trunc(value) != value))
            fail("bound type '" + type + "' on column '" + std::string(var) + "' requires an integral value", ln);
        double& lo = out_.var_lower[j];
        double& hi = out_.var_upper[j];
        int32_t& kind = out_.var_type[j];
        if (type == "LO") {
            lo = value;
            lower_explicit_[j] = 1;
        } else if (type == "UP") {
            hi = value;
            // A negative UP on a column whose lower bound is still the implicit
            // 0 opens the lower bound, as the reference (and common practice) do.
            if (value < 0.0 && !lower_explicit_[j] && lo == 0.0) {
                lo = -kInf;
                warn("negative UP bound on '" + std::string(var) + "' opened its lower bound to -infinity");
            }
        } else if (type == "FX") {
            lo = value;
            hi = value;
            lower_explicit_[j] = 1;
        } else if (type == "FR") {
            lo = -kInf;
            hi = kInf;
            lower_explicit_[j] = 1;
        } else if (type == "MI") {
            lo = -kInf;
            lower_explicit_[j] = 1;
        } else if (type == "PL") {
            hi = kInf;
        } else if (type == "BV") {
            lo = 0.0;
            hi = 1.0;
            kind = kBinary;
            lower_explicit_[j] = 1;
        } else if (type == "LI") {
            lo = value;
            lower_explicit_[j] = 1;
            if (kind == kContinuous) kind = kInteger;
        } else if (type == "UI") {
            hi = value;
            if (kind == kContinuous) kind = kInteger;
        } else {
            fail("unknown bound type '" + std::string(tok[0]) + "' on column '" + std::string(var) + "'", ln);
        }
    }

    void finish() {
        pdlpgpu_mps& m = out_;
        const size_t n = m.var_names.size(), rows = m.row_names.size();
        // Objective terms: one per column that appeared with the objective row,
        // its values summed from 0.0 in file order.
        for (size_t j = 0; j < n; ++j)
            if (obj_has_[j]) {
                m.obj_index.push_back(static_cast<int32_t>(j));
                m.obj_value.push_back(0.0 + obj_sum_[j]);
            }
        // Constraint terms: a stable counting sort by row over the segments in
        // file order, then per row by column (stable), duplicates summed from
        // 0.0 in file order.
        size_t nt = 0;
        for (const Segment& sg : segs_) nt += sg.row.size();
        std::vector<int64_t> start(rows + 1, 0);
        for (const Segment& sg : segs_)
            for (int32_t r : sg.row) ++start[static_cast<size_t>(r) + 1];
        for (size_t i = 0; i < rows; ++i) start[i + 1] += start[i];
        std::vector<int32_t> col(nt);
        std::vector<double> val(nt);
        {
            std::vector<int64_t> fill(start.begin(), start.end() - 1);
            for (Segment& sg : segs_) {
                for (size_t k = 0; k < sg.row.size(); ++k) {
                    const int64_t d = fill[static_cast<size_t>(sg.row[k])]++;
                    col[static_cast<size_t>(d)] = sg.col[k];
                    val[static_cast<size_t>(d)] = sg.val[k];
                }
                std::vector<int32_t>().swap(sg.row);
                std::vector<int32_t>().swap(sg.col);
                std::vector<double>().swap(sg.val);
            }
        }
        m.row_start.assign(rows + 1, 0);
        m.row_index.resize(nt);
        m.row_value.resize(nt);
        size_t w = 0;
        std::vector<size_t> order;
        for (size_t i = 0; i < rows; ++i) {
            const size_t b = static_cast<size_t>(start[i]), e = static_cast<size_t>(start[i + 1]);
            bool sorted = true;
            for (size_t k = b + 1; k < e && sorted; ++k) sorted = col[k - 1] < col[k];
            if (sorted) {
                for (size_t k = b; k < e; ++k, ++w) {
                    m.row_index[w] = col[k];
                    m.row_value[w] = 0.0 + val[k];
                }
            } else {
                order.resize(e - b);
                std::iota(order.begin(), order.end(), b);
                std::stable_sort(order.begin(), order.end(),
                                 [&](size_t x, size_t y) { return col[x] < col[y]; });
                for (size_t q = 0; q < order.size(); ++w) {
                    const int32_t c = col[order[q]];
                    double sum = 0.0;
                    for (; q < order.size() && col[order[q]] == c; ++q) sum += val[order[q]];
                    m.row_index[w] = c;
                    m.row_value[w] = sum;
                }
            }
            m.row_start[i + 1] = static_cast<int64_t>(w);
        }
        m.row_index.resize(w);
        m.row_value.resize(w);
        // Quadratic terms: by (i, j), summed in file order, zero sums dropped.
        std::vector<size_t> qo(q_lo_.size());
        std::iota(qo.begin(), qo.end(), size_t(0));
        std::stable_sort(qo.begin(), qo.end(), [&](size_t x, size_t y) {
            return q_lo_[x] != q_lo_[y] ? q_lo_[x] < q_lo_[y] : q_hi_[x] < q_hi_[y];
        });
        for (size_t q = 0; q < qo.size();) {
            const int32_t a = q_lo_[qo[q]], b = q_hi_[qo[q]];
            double sum = 0.0;
            for (; q < qo.size() && q_lo_[qo[q]] == a && q_hi_[qo[q]] == b; ++q) sum += q_val_[qo[q]];
            if (sum == 0.0) continue;
            m.q_i.push_back(a);
            m.q_j.push_back(b);
            m.q_value.push_back(sum);
        }
        m.offset = offset_;
        // Row bounds from sense, RHS and RANGES (finalizeRowBounds).
        m.row_lower.resize(rows);
        m.row_upper.resize(rows);
        for (size_t i = 0; i < rows; ++i) {
            const double r = rhs_[i];
            double& lo = m.row_lower[i];
            double& hi = m.row_upper[i];
            if (!has_range_[i]) {
                if (sense_[i] == kLess) { lo = -kInf; hi = r; }
                else if (sense_[i] == kGreater) { lo = r; hi = kInf; }
                else { lo = r; hi = r; }
                continue;
            }
            const double range = range_[i];
            const double width = std::abs(range);
            if (sense_[i] == kLess) { lo = r - width; hi = r; }
            else if (sense_[i] == kGreater) { lo = r; hi = r + width; }
            else if (range >= 0.0) { lo = r; hi = r + range; }
            else { lo = r + range; hi = r; }
        }
    }

    pdlpgpu_mps& out_;
    std::string buf_;
    Section section_ = Section::None;
    sv objective_;
    NameTable rows_, cols_, free_;
    sv last_col_name_;
    int32_t last_col_ = -1;
    bool integer_marker_ = false;
    sv rhs_vector_, ranges_vector_;
    std::vector<char> sense_, has_range_, lower_explicit_, obj_has_;
    std::vector<double> rhs_, range_, obj_sum_;
    double offset_ = 0.0;
    // Constraint terms in file order, as a list of segments: the sequential
    // reader appends to the last one, a parallel COLUMNS section adds its
    // chunks' arrays as they are.
    struct Segment {
        std::vector<int32_t> row, col;
        std::vector<double> val;
    };
    std::vector<Segment> segs_ = std::vector<Segment>(1);
    std::vector<int32_t> q_lo_, q_hi_;
    std::vector<double> q_val_;
    Pending pending_[kAhead];
    int pending_head_ = 0, pending_count_ = 0;
};

int fail_abi(const std::string& message) {
    pdlpgpu_internal_set_error(message.c_str());
    return -1;
}

// Appends text, integers and doubles (std::to_chars with precision 17 in
// general format, which is printf's %.17g) without temporary strings.
struct Out {
    std::string buf;
    Out& operator<<(sv t) {
        buf.append(t.data(), t.size());
        return *this;
    }
    Out& operator<<(char c) {
        buf.push_back(c);
        return *this;
    }
    Out& num(int64_t v) {
        char b[24];
        const auto r = std::to_chars(b, b + sizeof(b), v);
        buf.append(b, static_cast<size_t>(r.ptr - b));
        return *this;
    }
    Out& real(double v) {
        char b[40];
        const auto r = std::to_chars(b, b + sizeof(b), v, std::chars_format::general, 17);
        buf.append(b, static_cast<size_t>(r.ptr - b));
        return *this;
    }
};

}  // namespace
}  // namespace pdlpgpu

extern "C" int32_t pdlpgpu_mps_read(const char* path, pdlpgpu_mps** model) {
    if (path == nullptr || model == nullptr) return pdlpgpu::fail_abi("pdlpgpu_mps_read: NULL argument");
    *model = nullptr;
    auto* m = new pdlpgpu_mps;
    try {
        pdlpgpu::Reader(*m).read(path);
    } catch (const std::exception& e) {
        delete m;
        return pdlpgpu::fail_abi(e.what());
    }
    *model = m;
    return 0;
}

extern "C" void pdlpgpu_mps_free(pdlpgpu_mps* model) { delete model; }

extern "C" void pdlpgpu_mps_sizes(const pdlpgpu_mps* m, int64_t* sizes) {
    sizes[0] = static_cast<int64_t>(m->var_names.size());
    sizes[1] = static_cast<int64_t>(m->row_names.size());
    sizes[2] = static_cast<int64_t>(m->obj_index.size());
    sizes[3] = static_cast<int64_t>(m->row_index.size());
    sizes[4] = static_cast<int64_t>(m->q_value.size());
    sizes[5] = static_cast<int64_t>(m->warnings.size());
    sizes[6] = m->sense;
    int64_t integral = 0;
    for (int32_t t : m->var_type) integral += t != 0;
    sizes[7] = integral;
}

extern "C" const char* pdlpgpu_mps_name(const pdlpgpu_mps* m, int32_t kind, int64_t index) {
    const std::vector<std::string>* v = nullptr;
    switch (kind) {
        case 0: return m->name.c_str();
        case 1: v = &m->var_names; break;
        case 2: v = &m->row_names; break;
        case 3: v = &m->warnings; break;
        default: return nullptr;
    }
    if (index < 0 || index >= static_cast<int64_t>(v->size())) return nullptr;
    return (*v)[static_cast<size_t>(index)].c_str();
}

extern "C" void pdlpgpu_mps_model(const pdlpgpu_mps* m, double* objective_offset,
                                  int32_t* objective_index, double* objective_value,
                                  int32_t* var_type, double* var_lower, double* var_upper,
                                  double* row_lower, double* row_upper, int64_t* row_start,
                                  int32_t* row_index, double* row_value, int32_t* quadratic_i,
                                  int32_t* quadratic_j, double* quadratic_value) {
    auto put = [](auto* dst, const auto& src) {
        if (dst != nullptr) std::copy(src.begin(), src.end(), dst);
    };
    if (objective_offset != nullptr) *objective_offset = m->offset;
    put(objective_index, m->obj_index);
    put(objective_value, m->obj_value);
    put(var_type, m->var_type);
    put(var_lower, m->var_lower);
    put(var_upper, m->var_upper);
    put(row_lower, m->row_lower);
    put(row_upper, m->row_upper);
    put(row_start, m->row_start);
    put(row_index, m->row_index);
    put(row_value, m->row_value);
    put(quadratic_i, m->q_i);
    put(quadratic_j, m->q_j);
    put(quadratic_value, m->q_value);
}

// adapter::toCompiledLp (pdlp_adapter.cpp:21-189) with default AdapterOptions
// (integers refused, quadratic terms refused), then CompiledLp::validate.
extern "C" int32_t pdlpgpu_mps_lp(pdlpgpu_mps* m, pdlpgpu_lp* lp, int32_t* objective_negated) {
    using pdlpgpu::fail_abi;
    if (m == nullptr || lp == nullptr) return fail_abi("pdlpgpu_mps_lp: NULL argument");
    const int64_t n = static_cast<int64_t>(m->var_names.size());
    const int64_t rows = static_cast<int64_t>(m->row_names.size());
    if (n > INT32_MAX || rows > INT32_MAX) return fail_abi("pdlpgpu_mps_lp: model too large for int32 indices");
    if (!m->q_value.empty()) return fail_abi("model has quadratic objective terms; PDLP solves linear programs only");
    int64_t integral = 0;
    for (int32_t t : m->var_type) integral += t != 0;
    if (integral > 0) {
        std::ostringstream e;
        e << "model has " << integral
          << " integer variables; route it to branch-and-cut, or set "
             "relaxIntegrality to solve the LP relaxation deliberately";
        return fail_abi(e.str());
    }
    const bool maximise = m->sense == 1;
    const double sign = maximise ? -1.0 : 1.0;
    m->lp_objective.assign(static_cast<size_t>(n), 0.0);
    for (size_t k = 0; k < m->obj_index.size(); ++k)
        m->lp_objective[static_cast<size_t>(m->obj_index[k])] += sign * m->obj_value[k];
    const double offset = sign * m->offset;
    for (int64_t j = 0; j < n; ++j) {
        const size_t q = static_cast<size_t>(j);
        if (m->var_lower[q] > m->var_upper[q]) {
            std::ostringstream e;
            e << "variable " << j << " (" << m->var_names[q] << ") has lower bound " << m->var_lower[q]
              << " above upper bound " << m->var_upper[q];
            return fail_abi(e.str());
        }
    }
    for (int64_t i = 0; i < rows; ++i) {
        const size_t q = static_cast<size_t>(i);
        if (m->row_lower[q] > m->row_upper[q]) {
            std::ostringstream e;
            e << "constraint " << i << " (" << m->row_names[q] << ") has lower bound " << m->row_lower[q]
              << " above upper bound " << m->row_upper[q];
            return fail_abi(e.str());
        }
    }
    m->lp_start.assign(static_cast<size_t>(rows) + 1, 0);
    m->lp_index.clear();
    m->lp_value.clear();
    for (int64_t i = 0; i < rows; ++i) {
        for (int64_t k = m->row_start[static_cast<size_t>(i)]; k < m->row_start[static_cast<size_t>(i) + 1]; ++k) {
            const double v = m->row_value[static_cast<size_t>(k)];
            if (!std::isfinite(v)) {
                std::ostringstream e;
                e << "constraint " << i << " has a non-finite coefficient";
                return fail_abi(e.str());
            }
            // Terms below 1e-12 in magnitude are dropped (kZeroTolerance); the
            // rest are distinct columns in increasing order already, so the
            // rows are in SparseMatrix::fromTriplets' canonical form.
            if (std::abs(v) < 1e-12) continue;
            m->lp_index.push_back(m->row_index[static_cast<size_t>(k)]);
            m->lp_value.push_back(v);
        }
        m->lp_start[static_cast<size_t>(i) + 1] = static_cast<int64_t>(m->lp_index.size());
    }
    // CompiledLp::validate.
    if (!std::isfinite(offset)) return fail_abi("CompiledLp rejected the translation: Objective offset must be finite");
    for (int64_t j = 0; j < n; ++j) {
        const size_t q = static_cast<size_t>(j);
        if (!std::isfinite(m->lp_objective[q]) || std::isnan(m->var_lower[q]) || std::isnan(m->var_upper[q]))
            return fail_abi("CompiledLp rejected the translation: Invalid objective coefficient or variable bounds");
    }
    for (int64_t i = 0; i < rows; ++i) {
        const size_t q = static_cast<size_t>(i);
        if (std::isnan(m->row_lower[q]) || std::isnan(m->row_upper[q]))
            return fail_abi("CompiledLp rejected the translation: Invalid row bounds");
    }
    lp->num_rows = static_cast<int32_t>(rows);
    lp->num_cols = static_cast<int32_t>(n);
    lp->row_start = m->lp_start.data();
    lp->col_index = m->lp_index.data();
    lp->values = m->lp_value.data();
    lp->objective = m->lp_objective.data();
    lp->objective_offset = offset;
    lp->row_lower = m->row_lower.data();
    lp->row_upper = m->row_upper.data();
    lp->var_lower = m->var_lower.data();
    lp->var_upper = m->var_upper.data();
    if (objective_negated != nullptr) *objective_negated = maximise ? 1 : 0;
    return 0;
}

extern "C" int32_t pdlpgpu_mps_write(const char* path, const pdlpgpu_lp* lp, const char* name) {
    using pdlpgpu::fail_abi;
    if (path == nullptr || lp == nullptr) return fail_abi("pdlpgpu_mps_write: NULL argument");
    const int32_t m = lp->num_rows, n = lp->num_cols;
    if (m < 0 || n < 0) return fail_abi("pdlpgpu_mps_write: negative dimensions");
    for (int32_t i = 0; i < m; ++i)
        if (!std::isfinite(lp->row_lower[i]) && !std::isfinite(lp->row_upper[i]))
            return fail_abi("pdlpgpu_mps_write: row " + std::to_string(i) + " has no finite bound");
    const int64_t nnz = m > 0 ? lp->row_start[m] : 0;
    pdlpgpu::Out o;
    o.buf.reserve(static_cast<size_t>(40) * (static_cast<size_t>(n) * 2 + static_cast<size_t>(m) * 2 +
                                             static_cast<size_t>(nnz)));
    o << "NAME " << ((name != nullptr && name[0] != '\0') ? std::string_view(name) : std::string_view("LP"))
      << "\nROWS\n N obj\n";
    for (int32_t i = 0; i < m; ++i) {
        const double lo = lp->row_lower[i], hi = lp->row_upper[i];
        const char sense = (std::isfinite(lo) && lo == hi) ? 'E' : (!std::isfinite(lo) ? 'L' : 'G');
        o << ' ' << sense << " r";
        o.num(i) << '\n';
    }
    // Column-wise entries: the transpose of the CSR (stable, so rows ascend).
    std::vector<int64_t> cs(static_cast<size_t>(n) + 1, 0);
    for (int64_t k = 0; k < nnz; ++k) ++cs[static_cast<size_t>(lp->col_index[k]) + 1];
    for (int32_t j = 0; j < n; ++j) cs[static_cast<size_t>(j) + 1] += cs[static_cast<size_t>(j)];
    std::vector<int32_t> tr(static_cast<size_t>(nnz));
    std::vector<double> tv(static_cast<size_t>(nnz));
    {
        std::vector<int64_t> fill(cs.begin(), cs.end() - 1);
        for (int32_t i = 0; i < m; ++i)
            for (int64_t k = lp->row_start[i]; k < lp->row_start[i + 1]; ++k) {
                const int64_t d = fill[static_cast<size_t>(lp->col_index[k])]++;
                tr[static_cast<size_t>(d)] = i;
                tv[static_cast<size_t>(d)] = lp->values[k];
            }
    }
    o << "COLUMNS\n";
    for (int32_t j = 0; j < n; ++j) {
        // The objective entry first, even when zero, so every column is
        // declared in order.
        o << " x";
        o.num(j) << " obj ";
        o.real(lp->objective[j]) << '\n';
        for (int64_t k = cs[static_cast<size_t>(j)]; k < cs[static_cast<size_t>(j) + 1]; ++k) {
            o << " x";
            o.num(j) << " r";
            o.num(tr[static_cast<size_t>(k)]) << ' ';
            o.real(tv[static_cast<size_t>(k)]) << '\n';
        }
    }
    o << "RHS\n";
    if (lp->objective_offset != 0.0) {
        o << " rhs obj ";
        o.real(-lp->objective_offset) << '\n';
    }
    bool ranged = false;
    for (int32_t i = 0; i < m; ++i) {
        const double lo = lp->row_lower[i], hi = lp->row_upper[i];
        const double r = std::isfinite(lo) ? lo : hi;
        if (r != 0.0 || std::signbit(r)) {
            o << " rhs r";
            o.num(i) << ' ';
            o.real(r) << '\n';
        }
        ranged = ranged || (std::isfinite(lo) && std::isfinite(hi) && lo != hi);
    }
    if (ranged) {
        o << "RANGES\n";
        for (int32_t i = 0; i < m; ++i) {
            const double lo = lp->row_lower[i], hi = lp->row_upper[i];
            if (std::isfinite(lo) && std::isfinite(hi) && lo != hi) {
                o << " rng r";
                o.num(i) << ' ';
                o.real(hi - lo) << '\n';
            }
        }
    }
    o << "BOUNDS\n";
    for (int32_t j = 0; j < n; ++j) {
        const double lo = lp->var_lower[j], hi = lp->var_upper[j];
        auto head = [&](std::string_view type) -> pdlpgpu::Out& {
            o << ' ' << type << " bnd x";
            return o.num(j);
        };
        if (std::isfinite(lo) && lo == hi) {
            head("FX") << ' ';
            o.real(lo) << '\n';
            continue;
        }
        if (!std::isfinite(lo) && !std::isfinite(hi)) {
            head("FR") << '\n';
            continue;
        }
        // LO is written when the lower bound is not the default +0, and also
        // before a negative UP, which readers would otherwise take as opening
        // the default lower bound to -infinity.
        if (!std::isfinite(lo)) {
            head("MI") << '\n';
        } else if (lo != 0.0 || std::signbit(lo) || (std::isfinite(hi) && hi < 0.0)) {
            head("LO") << ' ';
            o.real(lo) << '\n';
        }
        if (std::isfinite(hi)) {
            head("UP") << ' ';
            o.real(hi) << '\n';
        }
    }
    o << "ENDATA\n";
    FILE* f = std::fopen(path, "wb");
    if (f == nullptr) return fail_abi(std::string("pdlpgpu_mps_write: cannot open ") + path);
    const size_t wrote = std::fwrite(o.buf.data(), 1, o.buf.size(), f);
    const bool closed = std::fclose(f) == 0;
    if (wrote != o.buf.size() || !closed) return fail_abi(std::string("pdlpgpu_mps_write: write failed for ") + path);
    return 0;
}
