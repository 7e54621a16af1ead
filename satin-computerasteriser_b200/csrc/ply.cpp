// PLY point-cloud input (PLYPointCloudLoader.swift:33-369), parsed on all
// host cores.
//
// The header rules, the vertex property semantics, the scalar conversions,
// the colour normalisation and the error cases follow the reference loader:
//   * the header ends at the first "end_header" in the data, followed by an
//     optional CR and an optional LF (:171-191); it must be valid UTF-8;
//   * header lines split at newlines, words at spaces, empty ones dropped
//     (:203-205); "format" ascii | binary_little_endian (:211-217);
//     "element vertex N" (:218-224); "property <type> <name>" inside the
//     vertex element, list properties rejected (:225-233);
//   * x, y, z are required; red/r/diffuse_red (and green, blue) are the
//     colour; every other property is read and ignored (:150-171);
//   * colour = clamp(value / scale(type), 0, 1) for integer types,
//     clamp(value, 0, 1) for floats; alpha is always 1; points without colour
//     properties are white (:307-330);
//   * ASCII: the body (valid UTF-8) splits into non-empty lines, each into
//     space-separated values parsed as the nearest float, with
//     truncatedBody when there are fewer lines than vertices or fewer values
//     than properties on a vertex line, and invalidASCIIValue(line, property)
//     for the first value that is not a number (:245-278);
//   * binary little-endian: stride = sum of the property sizes, truncatedBody
//     if the body is shorter than count * stride (:280-305), each scalar
//     converted to float with round-to-nearest (:332-352).
// The body is split into one range per thread: the binary body by vertex,
// the ASCII body at line boundaries after a parallel line count.  Errors are
// those of the reference's sequential loop: the lowest failing line wins.
#include <fcntl.h>
#include <locale.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <strings.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <limits>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "cr_internal.h"

using cri::fail;

namespace {

enum PlyType { T_I8, T_U8, T_I16, T_U16, T_I32, T_U32, T_F32, T_F64 };
enum Sem { S_X, S_Y, S_Z, S_R, S_G, S_B, S_IGNORED };

struct Field {
    Sem sem;
    std::string name;
    PlyType type;
    uint32_t offset;
};

struct Header {
    uint32_t format = 0;  // 0 ascii, 1 binary_little_endian
    uint64_t count = 0;
    std::vector<Field> fields;
    uint32_t stride = 0;
    uint64_t body = 0;
};

bool type_of(const std::string &s, PlyType &t) {  // PLYScalarType.init (:69-80)
    if (s == "char" || s == "int8") t = T_I8;
    else if (s == "uchar" || s == "uint8") t = T_U8;
    else if (s == "short" || s == "int16") t = T_I16;
    else if (s == "ushort" || s == "uint16") t = T_U16;
    else if (s == "int" || s == "int32") t = T_I32;
    else if (s == "uint" || s == "uint32") t = T_U32;
    else if (s == "float" || s == "float32") t = T_F32;
    else if (s == "double" || s == "float64") t = T_F64;
    else return false;
    return true;
}

uint32_t type_bytes(PlyType t) {
    switch (t) {
    case T_I8: case T_U8: return 1;
    case T_I16: case T_U16: return 2;
    case T_F64: return 8;
    default: return 4;
    }
}

float color_scale(PlyType t) {  // PLYScalarType.colorScale (:93-103)
    switch (t) {
    case T_I8: return 127.0f;
    case T_U8: return 255.0f;
    case T_I16: return 32767.0f;
    case T_U16: return 65535.0f;
    case T_I32: return 2147483647.0f;
    case T_U32: return 4294967295.0f;
    default: return 1.0f;
    }
}

Sem sem_of(const std::string &n) {  // semantic(for:) (:160-170)
    if (n == "x") return S_X;
    if (n == "y") return S_Y;
    if (n == "z") return S_Z;
    if (n == "red" || n == "r" || n == "diffuse_red") return S_R;
    if (n == "green" || n == "g" || n == "diffuse_green") return S_G;
    if (n == "blue" || n == "b" || n == "diffuse_blue") return S_B;
    return S_IGNORED;
}

// Length of the newline code point at p (0 if none): LF, VT, FF, CR, NEL,
// LINE SEPARATOR, PARAGRAPH SEPARATOR (Character.isNewline).
inline size_t newline_at(const uint8_t *p, const uint8_t *end) {
    const uint8_t c = *p;
    if (c >= 0x0A && c <= 0x0D) return 1;
    if (c == 0xC2 && p + 1 < end && p[1] == 0x85) return 2;
    if (c == 0xE2 && p + 2 < end && p[1] == 0x80 && (p[2] == 0xA8 || p[2] == 0xA9)) return 3;
    return 0;
}

// Well-formed UTF-8 (no overlong forms, surrogates or values above U+10FFFF).
bool valid_utf8(const uint8_t *p, const uint8_t *end) {
    while (p < end) {
        const uint8_t c = *p;
        if (c < 0x80) {
            ++p;
            continue;
        }
        int n;
        uint32_t cp;
        if ((c & 0xE0) == 0xC0) n = 1, cp = c & 0x1F;
        else if ((c & 0xF0) == 0xE0) n = 2, cp = c & 0x0F;
        else if ((c & 0xF8) == 0xF0) n = 3, cp = c & 0x07;
        else return false;
        if (end - p <= n) return false;
        for (int k = 1; k <= n; ++k) {
            if ((p[k] & 0xC0) != 0x80) return false;
            cp = (cp << 6) | (p[k] & 0x3F);
        }
        if ((n == 1 && cp < 0x80) || (n == 2 && cp < 0x800) || (n == 3 && cp < 0x10000) ||
            cp > 0x10FFFF || (cp >= 0xD800 && cp <= 0xDFFF))
            return false;
        p += n + 1;
    }
    return true;
}

// Swift Int(String): optional sign, decimal digits, no overflow.
bool parse_int(const std::string &s, int64_t &out) {
    size_t i = 0;
    bool neg = false;
    if (i < s.size() && (s[i] == '+' || s[i] == '-')) neg = s[i++] == '-';
    if (i == s.size()) return false;
    uint64_t v = 0;
    for (; i < s.size(); ++i) {
        if (s[i] < '0' || s[i] > '9') return false;
        if (v > (uint64_t)INT64_MAX / 10) return false;
        v = v * 10 + (uint64_t)(s[i] - '0');
        if (v > (uint64_t)INT64_MAX + (neg ? 1 : 0)) return false;
    }
    out = neg ? (int64_t)(0 - v) : (int64_t)v;
    return true;
}

std::vector<std::string> split_spaces(const uint8_t *b, const uint8_t *e) {
    std::vector<std::string> out;
    const uint8_t *p = b;
    while (p < e) {
        while (p < e && *p == ' ') ++p;
        const uint8_t *q = p;
        while (q < e && *q != ' ') ++q;
        if (q > p) out.emplace_back((const char *)p, (size_t)(q - p));
        p = q;
    }
    return out;
}

cr_status parse_header(const uint8_t *d, uint64_t n, Header &h) {  // parseHeader (:171-240)
    if (n < 4) return fail(CR_ERR_FORMAT, "invalidHeader");
    static const char kMarker[] = "end_header";
    const size_t m = sizeof(kMarker) - 1;
    const uint8_t *hit = nullptr;
    if (n >= m) {
        const uint8_t *p = d, *last = d + (n - m);
        while (p <= last) {
            p = (const uint8_t *)std::memchr(p, 'e', (size_t)(last - p) + 1);
            if (!p) break;
            if (std::memcmp(p, kMarker, m) == 0) {
                hit = p;
                break;
            }
            ++p;
        }
    }
    if (!hit) return fail(CR_ERR_FORMAT, "invalidHeader");
    uint64_t body = (uint64_t)(hit - d) + m;
    if (body < n && d[body] == 13) ++body;
    if (body < n && d[body] == 10) ++body;
    if (!valid_utf8(d, d + body)) return fail(CR_ERR_FORMAT, "invalidHeader");

    bool have_format = false, have_count = false, in_vertex = false;
    const uint8_t *p = d, *end = d + body;
    while (p < end) {
        const uint8_t *q = p;
        size_t nl = 0;
        while (q < end && (nl = newline_at(q, end)) == 0) ++q;
        const std::vector<std::string> parts = split_spaces(p, q);
        p = q < end ? q + nl : end;
        if (parts.empty()) continue;
        const std::string &k = parts[0];
        if (k == "format") {
            if (parts.size() < 3) return fail(CR_ERR_FORMAT, "invalidHeader");
            if (parts[1] == "ascii") h.format = 0;
            else if (parts[1] == "binary_little_endian") h.format = 1;
            else return fail(CR_ERR_FORMAT, "unsupportedFormat(" + parts[1] + ")");
            have_format = true;
        } else if (k == "element") {
            if (parts.size() < 3) return fail(CR_ERR_FORMAT, "invalidHeader");
            in_vertex = parts[1] == "vertex";
            if (in_vertex) {
                int64_t c;
                // A negative count traps in the reference's loops; rejected here.
                if (!parse_int(parts[2], c) || c < 0) return fail(CR_ERR_FORMAT, "invalidHeader");
                h.count = (uint64_t)c;
                have_count = true;
            }
        } else if (k == "property" && in_vertex) {
            if (parts.size() < 3) return fail(CR_ERR_FORMAT, "invalidHeader");
            if (parts[1] == "list") {
                std::string rest;
                for (size_t i = 2; i < parts.size(); ++i) rest += (i > 2 ? " " : "") + parts[i];
                return fail(CR_ERR_FORMAT, "unsupportedProperty(list " + rest + ")");
            }
            PlyType t;
            if (!type_of(parts[1], t)) return fail(CR_ERR_FORMAT, "unsupportedProperty(" + parts[1] + ")");
            h.fields.push_back(Field{sem_of(parts[2]), parts[2], t, 0});
        }
    }
    if (!have_format) return fail(CR_ERR_FORMAT, "invalidHeader");
    if (!have_count) return fail(CR_ERR_FORMAT, "missingVertexElement");
    // PLYVertexLayout (:140-158).
    uint32_t off = 0;
    bool x = false, y = false, z = false;
    for (Field &f : h.fields) {
        f.offset = off;
        off += type_bytes(f.type);
        x |= f.sem == S_X;
        y |= f.sem == S_Y;
        z |= f.sem == S_Z;
    }
    if (!(x && y && z)) return fail(CR_ERR_FORMAT, "missingProperty(x, y, z)");
    h.stride = off;
    h.body = body;
    return CR_OK;
}

inline float norm_color(float v, PlyType t) {  // normalizedColor (:320-325)
    const float x = (t == T_F32 || t == T_F64) ? v : v / color_scale(t);
    return std::fmin(std::fmax(x, 0.0f), 1.0f);
}

// assign(value:field:position:color:) (:307-318).
inline void assign(float v, const Field &f, float *pos, float *col) {
    switch (f.sem) {
    case S_X: pos[0] = v; break;
    case S_Y: pos[1] = v; break;
    case S_Z: pos[2] = v; break;
    case S_R: col[0] = norm_color(v, f.type); break;
    case S_G: col[1] = norm_color(v, f.type); break;
    case S_B: col[2] = norm_color(v, f.type); break;
    default: break;
    }
}

inline uint32_t rd32(const uint8_t *b) {
    return (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
}

inline float read_scalar(PlyType t, const uint8_t *b) {  // readScalar (:327-349)
    switch (t) {
    case T_I8: return (float)(int8_t)b[0];
    case T_U8: return (float)b[0];
    case T_I16: return (float)(int16_t)(uint16_t)(b[0] | (b[1] << 8));
    case T_U16: return (float)(uint16_t)(b[0] | (b[1] << 8));
    case T_I32: return (float)(int32_t)rd32(b);
    case T_U32: return (float)rd32(b);
    case T_F32: {
        const uint32_t u = rd32(b);
        float f;
        std::memcpy(&f, &u, 4);
        return f;
    }
    default: {
        const uint64_t u = (uint64_t)rd32(b) | ((uint64_t)rd32(b + 4) << 32);
        double x;
        std::memcpy(&x, &u, 8);
        return (float)x;
    }
    }
}

int thread_count(int threads) {
    if (threads > 0) return threads;
    const unsigned hc = std::thread::hardware_concurrency();
    return hc ? (int)hc : 1;
}

template <typename F>
void run_parallel(int nt, F &&f) {
    if (nt <= 1) {
        f(0);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(f, t);
    f(0);
    for (auto &th : pool) th.join();
}

// Float(Substring) as Swift's standard library parses it: the token as a C
// string (it ends at a NUL byte), no leading whitespace, strtof in the C
// locale (nearest float; decimal, hexadecimal, inf, nan), "snan" with an
// optional sign as a signalling NaN, and no result when strtof reports a
// range error with an infinite or zero result.
locale_t c_locale() {
    static locale_t loc = newlocale(LC_ALL_MASK, "C", (locale_t)0);
    return loc;
}

inline bool parse_float(const uint8_t *b, const uint8_t *e, float &out) {
    char buf[96];
    std::string big;
    const size_t n = (size_t)(e - b);
    const char *s;
    if (n < sizeof(buf)) {
        std::memcpy(buf, b, n);
        buf[n] = 0;
        s = buf;
    } else {
        big.assign((const char *)b, n);
        s = big.c_str();
    }
    const unsigned char c0 = (unsigned char)s[0];
    if (c0 == 0 || (c0 >= 9 && c0 <= 13) || c0 == 32) return false;
    const char *t = (s[0] == '+' || s[0] == '-') ? s + 1 : s;
    if (strcasecmp(t, "snan") == 0) {
        out = s[0] == '-' ? -std::numeric_limits<float>::signaling_NaN()
                          : std::numeric_limits<float>::signaling_NaN();
        return true;
    }
    char *endp = nullptr;
    errno = 0;
    out = strtof_l(s, &endp, c_locale());
    if (errno == ERANGE && (std::isinf(out) || out == 0.0f)) return false;
    return *endp == 0;
}

struct AsciiError {
    uint64_t line = UINT64_MAX;  // vertex line index (0-based)
    int kind = 0;                // 1 truncatedBody, 2 invalidASCIIValue
    std::string property;
};

cr_status parse_ascii(const uint8_t *d, uint64_t n, const Header &h, int nt, float *pos,
                      float *col) {
    const uint8_t *body = d + h.body, *end = d + n;
    const uint64_t bytes = (uint64_t)(end - body);
    nt = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)nt, bytes / 65536 + 1));
    // Range starts just after an LF byte (a line boundary; an LF never sits
    // inside a multi-byte sequence).
    std::vector<const uint8_t *> cut(nt + 1);
    cut[0] = body;
    cut[nt] = end;
    for (int t = 1; t < nt; ++t) {
        const uint8_t *p = body + bytes * (uint64_t)t / (uint64_t)nt;
        p = std::max(p, cut[t - 1]);
        const uint8_t *lf = (const uint8_t *)std::memchr(p, '\n', (size_t)(end - p));
        cut[t] = lf ? lf + 1 : end;
    }
    // Pass 1: UTF-8 check and non-empty line count per range.
    std::vector<uint64_t> lines(nt, 0);
    std::vector<char> ok(nt, 1);
    run_parallel(nt, [&](int t) {
        const uint8_t *p = cut[t], *e = cut[t + 1];
        if (!valid_utf8(p, e)) {
            ok[t] = 0;
            return;
        }
        uint64_t c = 0;
        while (p < e) {
            const uint8_t *q = p;
            size_t nl = 0;
            while (q < e && (nl = newline_at(q, end)) == 0) ++q;
            if (q > p) ++c;
            p = q < e ? q + nl : e;
        }
        lines[t] = c;
    });
    for (int t = 0; t < nt; ++t)
        if (!ok[t]) return fail(CR_ERR_FORMAT, "truncatedBody");
    uint64_t total = 0;
    std::vector<uint64_t> first(nt);
    for (int t = 0; t < nt; ++t) {
        first[t] = total;
        total += lines[t];
    }
    if (total < h.count) return fail(CR_ERR_FORMAT, "truncatedBody");
    // Pass 2: the first h.count lines, each range from its first line index.
    const size_t nf = h.fields.size();
    std::vector<AsciiError> err(nt);
    run_parallel(nt, [&](int t) {
        uint64_t g = first[t];
        if (g >= h.count) return;
        const uint8_t *p = cut[t], *e = cut[t + 1];
        std::vector<std::pair<const uint8_t *, const uint8_t *>> tok;
        tok.reserve(nf + 4);
        while (p < e && g < h.count) {
            const uint8_t *q = p;
            size_t nl = 0;
            while (q < e && (nl = newline_at(q, end)) == 0) ++q;
            const uint8_t *lb = p, *le = q;
            p = q < e ? q + nl : e;
            if (le == lb) continue;
            tok.clear();
            for (const uint8_t *a = lb; a < le;) {
                while (a < le && *a == ' ') ++a;
                const uint8_t *z = a;
                while (z < le && *z != ' ') ++z;
                if (z > a) tok.emplace_back(a, z);
                a = z;
            }
            if (tok.size() < nf) {
                err[t] = AsciiError{g, 1, ""};
                return;
            }
            float *po = pos + 4 * g, *co = col + 4 * g;
            po[0] = po[1] = po[2] = 0.0f;
            po[3] = 1.0f;
            co[0] = co[1] = co[2] = co[3] = 1.0f;
            for (size_t f = 0; f < nf; ++f) {
                float v;
                if (!parse_float(tok[f].first, tok[f].second, v)) {
                    err[t] = AsciiError{g, 2, h.fields[f].name};
                    return;
                }
                assign(v, h.fields[f], po, co);
            }
            ++g;
        }
    });
    const AsciiError *worst = nullptr;
    for (const AsciiError &e : err)
        if (e.kind && (!worst || e.line < worst->line)) worst = &e;
    if (worst) {
        if (worst->kind == 1) return fail(CR_ERR_FORMAT, "truncatedBody");
        return fail(CR_ERR_FORMAT, "invalidASCIIValue(line: " + std::to_string(worst->line + 1) +
                                       ", property: " + worst->property + ")");
    }
    return CR_OK;
}

cr_status parse_binary(const uint8_t *d, uint64_t n, const Header &h, int nt, float *pos,
                       float *col) {
    const uint64_t need = h.count * (uint64_t)h.stride;
    if (h.stride && need / h.stride != h.count) return fail(CR_ERR_FORMAT, "truncatedBody");
    if (h.body + need > n) return fail(CR_ERR_FORMAT, "truncatedBody");
    nt = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)nt, h.count / 4096 + 1));
    run_parallel(nt, [&](int t) {
        const uint64_t v0 = h.count * (uint64_t)t / (uint64_t)nt;
        const uint64_t v1 = h.count * (uint64_t)(t + 1) / (uint64_t)nt;
        for (uint64_t v = v0; v < v1; ++v) {
            const uint8_t *vb = d + h.body + v * h.stride;
            float *po = pos + 4 * v, *co = col + 4 * v;
            po[0] = po[1] = po[2] = 0.0f;
            po[3] = 1.0f;
            co[0] = co[1] = co[2] = co[3] = 1.0f;
            for (const Field &f : h.fields) assign(read_scalar(f.type, vb + f.offset), f, po, co);
        }
    });
    return CR_OK;
}

void fill_header(const Header &h, cr_ply_header *out) {
    out->vertexCount = h.count;
    out->bodyOffset = h.body;
    out->format = h.format;
    out->propertyCount = (uint32_t)h.fields.size();
    out->stride = h.stride;
    uint32_t nc = 0;
    for (const Field &f : h.fields) nc += (f.sem == S_R || f.sem == S_G || f.sem == S_B) ? 1 : 0;
    out->colorProperties = nc;
}

}  // namespace

extern "C" {

CR_API cr_status cr_ply_read_header(const uint8_t *data, uint64_t size, cr_ply_header *out) {
    if (!out || (!data && size)) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    Header h;
    cr_status st = parse_header(data, size, h);
    if (st) return st;
    // A body that cannot hold the vertices (each ASCII vertex needs a
    // non-empty line; each binary vertex `stride` bytes) is truncatedBody
    // before anything is sized from the count.
    const uint64_t body = size - h.body;
    if (h.format == 0 ? h.count > body
                      : (h.count && (h.count > body / h.stride)))
        return fail(CR_ERR_FORMAT, "truncatedBody");
    fill_header(h, out);
    return CR_OK;
}

CR_API cr_status cr_ply_parse(const uint8_t *data, uint64_t size, int threads, float *positions,
                              float *colors) {
    if (!data && size) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    Header h;
    cr_status st = parse_header(data, size, h);
    if (st) return st;
    if (h.count && (!positions || !colors))
        return fail(CR_ERR_INVALID_ARGUMENT, "positions / colors is null");
    const int nt = thread_count(threads);
    return h.format == 0 ? parse_ascii(data, size, h, nt, positions, colors)
                         : parse_binary(data, size, h, nt, positions, colors);
}

CR_API cr_status cr_file_map(const char *path, const uint8_t **data, uint64_t *size) {
    if (!path || !data || !size) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    *data = nullptr;
    *size = 0;
    const int fd = open(path, O_RDONLY);
    if (fd < 0) return fail(CR_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
    struct stat sb;
    if (fstat(fd, &sb) != 0) {
        close(fd);
        return fail(CR_ERR_INVALID_ARGUMENT, std::string("cannot stat ") + path);
    }
    if (sb.st_size == 0) {
        close(fd);
        return CR_OK;
    }
    void *p = mmap(nullptr, (size_t)sb.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);
    if (p == MAP_FAILED) return fail(CR_ERR_OUT_OF_MEMORY, std::string("cannot map ") + path);
    madvise(p, (size_t)sb.st_size, MADV_SEQUENTIAL);
    *data = (const uint8_t *)p;
    *size = (uint64_t)sb.st_size;
    return CR_OK;
}

CR_API cr_status cr_file_unmap(const uint8_t *data, uint64_t size) {
    if (data && size) munmap((void *)data, (size_t)size);
    return CR_OK;
}

}  // extern "C"
