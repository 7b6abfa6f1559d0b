// ply.cpp - the Gaussian model's on-disk form: the 3D Gaussian Splatting PLY layout (writer and
// reader) and plain point clouds read as small opaque Gaussians. Host code, run once per model.
//
// Behaviour follows writeSplatPly / readSplatPly (engine/src/splat/SplatPly.cpp:261-342): the writer's
// header text and record layout are the format contract (x y z nx ny nz f_dc_0..2 opacity scale_0..2
// rot_0..3, float32 little endian); the reader accepts ASCII and both binary byte orders, keeps only
// vertices with finite x/y/z, treats a file with f_dc_0, opacity, scale_0 and rot_0 as Gaussians
// (absent sibling columns read as NaN) and anything else with x/y/z as a point cloud (8- and 16-bit
// colours scaled to 0..1, grey 0.8 without colours; Gaussians from initGaussiansFromPoints with
// opacity logit(0.95) and scales halved).
//
// The reader is organised around the header's byte layout rather than a value stream: the header
// becomes one record layout per element (each scalar property's byte offset inside a record, and the
// record size when no property is a list). Binary vertex tables with fixed-size records, which is
// every file the writer and common splat tools produce, are decoded column by column straight from
// their byte offsets; ASCII bodies and records with list properties go through a token / byte cursor.

#include "host_io.h"

#include <array>
#include <charconv>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iterator>

namespace u3dg {

namespace {

bool fail(std::string *error, const std::string &m)
{
    if (error)
        *error = m;
    return false;
}

bool hostLittleEndian()
{
    const uint32_t probe = 1;
    uint8_t first;
    std::memcpy(&first, &probe, 1);
    return first == 1;
}

// ---------------------------------------------------------------- header layout

// One PLY scalar encoding: size in bytes, integer or IEEE float, signedness.
struct Scalar {
    uint8_t bytes = 0;
    bool real = false;
    bool sign = false;
};

bool scalarNamed(const std::string &s, Scalar &t)
{
    // PLY 1.0 names and their sized aliases.
    struct Entry {
        const char *a, *b;
        Scalar t;
    };
    static const Entry table[] = {
        {"char", "int8", {1, false, true}},    {"uchar", "uint8", {1, false, false}},
        {"short", "int16", {2, false, true}},  {"ushort", "uint16", {2, false, false}},
        {"int", "int32", {4, false, true}},    {"uint", "uint32", {4, false, false}},
        {"float", "float32", {4, true, true}}, {"double", "float64", {8, true, true}},
    };
    for (const Entry &e : table)
        if (s == e.a || s == e.b) {
            t = e.t;
            return true;
        }
    return false;
}

// A property of an element: a scalar at a byte offset of a fixed-size record, or a list.
struct Property {
    std::string name;
    Scalar value;
    bool list = false;
    Scalar length; // list length encoding
    size_t offset = 0; // within the record (meaningful while the element has fixed-size records)
};

struct Element {
    std::string name;
    size_t count = 0;
    std::vector<Property> props;
    bool fixedSize = true; // no list property
    size_t recordBytes = 0; // record size when fixedSize
};

enum class Encoding { Ascii, BinaryLittle, BinaryBig };

struct Header {
    Encoding encoding = Encoding::Ascii;
    std::vector<Element> elements;
    size_t bodyStart = 0; // byte after the end_header line
};

// Splits one header line into whitespace-separated words.
std::vector<std::string> words(const char *b, const char *e)
{
    std::vector<std::string> out;
    while (b < e) {
        while (b < e && std::isspace(static_cast<unsigned char>(*b)))
            ++b;
        const char *s = b;
        while (b < e && !std::isspace(static_cast<unsigned char>(*b)))
            ++b;
        if (b > s)
            out.emplace_back(s, b);
    }
    return out;
}

bool parseHeader(const std::vector<char> &file, Header &h, std::string *error)
{
    const char *const base = file.data();
    const size_t size = file.size();
    if (size < 3 || std::memcmp(base, "ply", 3) != 0)
        return fail(error, "Not a PLY file");
    size_t pos = 0;
    bool ended = false;
    while (pos < size && !ended) {
        const void *nl = std::memchr(base + pos, '\n', size - pos);
        if (!nl)
            return fail(error, "PLY header is not terminated by an end_header line");
        const size_t lineEnd = size_t(static_cast<const char *>(nl) - base);
        const std::vector<std::string> w = words(base + pos, base + lineEnd);
        pos = lineEnd + 1;
        if (w.empty())
            continue;
        const std::string &key = w[0];
        if (key == "end_header") {
            ended = true;
        } else if (key == "format") {
            if (w.size() < 2)
                return fail(error, "PLY format line without a format");
            if (w[1] == "ascii")
                h.encoding = Encoding::Ascii;
            else if (w[1] == "binary_little_endian")
                h.encoding = Encoding::BinaryLittle;
            else if (w[1] == "binary_big_endian")
                h.encoding = Encoding::BinaryBig;
            else
                return fail(error, "Unknown PLY format " + w[1]);
        } else if (key == "element") {
            Element e;
            if (w.size() >= 2)
                e.name = w[1];
            if (w.size() >= 3) {
                unsigned long long c = 0;
                const auto r = std::from_chars(w[2].data(), w[2].data() + w[2].size(), c);
                if (r.ec != std::errc())
                    return fail(error, "PLY element count is not a number: " + w[2]);
                e.count = size_t(c);
            }
            h.elements.push_back(std::move(e));
        } else if (key == "property" && !h.elements.empty()) {
            Property p;
            bool ok;
            if (w.size() >= 2 && w[1] == "list") {
                p.list = true;
                ok = w.size() >= 5 && scalarNamed(w[2], p.length) && scalarNamed(w[3], p.value);
                if (ok)
                    p.name = w[4];
            } else {
                ok = w.size() >= 3 && scalarNamed(w[1], p.value);
                if (ok)
                    p.name = w[2];
            }
            if (!ok) {
                std::string line = "property";
                for (size_t k = 1; k < w.size(); ++k)
                    line += " " + w[k];
                return fail(error, "Unsupported PLY property: " + line);
            }
            Element &e = h.elements.back();
            p.offset = e.recordBytes;
            if (p.list)
                e.fixedSize = false;
            else
                e.recordBytes += p.value.bytes;
            e.props.push_back(std::move(p));
        }
        // comment, obj_info and unknown keywords carry nothing the reader needs.
    }
    if (!ended)
        return fail(error, "PLY header is not terminated by an end_header line");
    h.bodyStart = pos;
    return true;
}

// ---------------------------------------------------------------- body decoding

// A binary scalar at p (in the file's byte order) as a double.
double decodeBinary(const unsigned char *p, Scalar t, bool swap)
{
    unsigned char b[8];
    std::memcpy(b, p, t.bytes);
    if (swap)
        for (int i = 0, j = t.bytes - 1; i < j; ++i, --j)
            std::swap(b[i], b[j]);
    // b now holds the value in host byte order.
    switch (t.bytes) {
    case 1: return t.sign ? double(int8_t(b[0])) : double(b[0]);
    case 2: {
        uint16_t u;
        std::memcpy(&u, b, 2);
        return t.sign ? double(int16_t(u)) : double(u);
    }
    case 4: {
        if (t.real) {
            float f;
            std::memcpy(&f, b, 4);
            return double(f);
        }
        uint32_t u;
        std::memcpy(&u, b, 4);
        return t.sign ? double(int32_t(u)) : double(u);
    }
    default: {
        double d;
        std::memcpy(&d, b, 8);
        return d;
    }
    }
}

// Sequential reader of values: whitespace-separated tokens (ASCII) or packed scalars (binary).
class Cursor
{
public:
    Cursor(const char *p, const char *end, Encoding enc) : p_(p), end_(end), enc_(enc) {}

    bool read(Scalar t, double &v)
    {
        if (enc_ == Encoding::Ascii)
            return token(v);
        if (size_t(end_ - p_) < t.bytes)
            return false;
        v = decodeBinary(reinterpret_cast<const unsigned char *>(p_), t, swap());
        p_ += t.bytes;
        return true;
    }

    bool skip(const Property &q)
    {
        double v;
        if (!q.list)
            return read(q.value, v);
        double n;
        if (!read(q.length, n) || !(n >= 0))
            return false;
        if (enc_ != Encoding::Ascii) {
            const double bytes = n * q.value.bytes;
            if (bytes > double(end_ - p_))
                return false;
            p_ += size_t(bytes);
            return true;
        }
        for (size_t k = 0; k < size_t(n); ++k)
            if (!token(v))
                return false;
        return true;
    }

    bool skipRecords(const Element &e)
    {
        if (enc_ != Encoding::Ascii && e.fixedSize) {
            const double bytes = double(e.count) * double(e.recordBytes);
            if (bytes > double(end_ - p_))
                return false;
            p_ += size_t(bytes);
            return true;
        }
        for (size_t i = 0; i < e.count; ++i)
            for (const Property &q : e.props)
                if (!skip(q))
                    return false;
        return true;
    }

    const char *position() const { return p_; }
    size_t remaining() const { return size_t(end_ - p_); }
    bool swap() const { return (enc_ == Encoding::BinaryLittle) != hostLittleEndian(); }

private:
    bool token(double &v)
    {
        while (p_ < end_ && std::isspace(static_cast<unsigned char>(*p_)))
            ++p_;
        const char *s = p_;
        while (p_ < end_ && !std::isspace(static_cast<unsigned char>(*p_)))
            ++p_;
        if (p_ == s)
            return false;
        // Decimal numbers only, read as far as they go (a stream extraction of a double does the same):
        // an optional sign, then a digit or a point; words such as nan or inf are not numbers here.
        if (*s == '+' && p_ - s > 1)
            ++s;
        const char *d = (*s == '-') ? s + 1 : s;
        if (d == p_ || !(std::isdigit(static_cast<unsigned char>(*d)) || *d == '.'))
            return false;
        const auto r = std::from_chars(s, p_, v);
        return r.ec == std::errc();
    }

    const char *p_, *end_;
    Encoding enc_;
};

// Vertex columns the model is built from, in this order.
enum Column { X, Y, Z, DC0, DC1, DC2, OPACITY, SCALE0, SCALE1, SCALE2, ROT0, ROT1, ROT2, ROT3, RED, GREEN, BLUE, kColumns };
const char *const kColumnName[kColumns] = {"x",       "y",       "z",       "f_dc_0", "f_dc_1", "f_dc_2",
                                            "opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1",
                                            "rot_2",   "rot_3",   "red",     "green",  "blue"};

struct VertexColumns {
    size_t count = 0;
    std::array<bool, kColumns> present{};
    std::array<std::vector<float>, kColumns> data; // count values each; NaN where the column is absent
};

// Divisor that maps an integer colour encoding to 0..1 (8 and 16 bits), or 1.
double colourScale(Column c, Scalar t)
{
    if ((c != RED && c != GREEN && c != BLUE) || t.real || t.sign)
        return 1.0;
    return t.bytes == 1 ? 255.0 : (t.bytes == 2 ? 65535.0 : 1.0);
}

bool decodeVertices(const std::vector<char> &file, const Header &h, VertexColumns &out, std::string *error)
{
    const char *end = file.data() + file.size();
    Cursor cur(file.data() + h.bodyStart, end, h.encoding);
    for (const Element &e : h.elements) {
        if (e.name != "vertex") {
            if (!cur.skipRecords(e))
                return fail(error, "Truncated PLY data in element " + e.name);
            continue;
        }
        // Which property feeds which column (the last property of a name wins, like a table fill).
        std::vector<int> target(e.props.size(), -1);
        for (size_t q = 0; q < e.props.size(); ++q)
            if (!e.props[q].list)
                for (int c = 0; c < kColumns; ++c)
                    if (e.props[q].name == kColumnName[c])
                        target[q] = c;
        out.count = e.count;
        for (int c = 0; c < kColumns; ++c) {
            out.present[size_t(c)] = false;
            out.data[size_t(c)].assign(e.count, std::nanf(""));
        }
        for (size_t q = 0; q < e.props.size(); ++q)
            if (target[q] >= 0)
                out.present[size_t(target[q])] = true;

        if (h.encoding != Encoding::Ascii && e.fixedSize) {
            // Column-wise decode straight from each property's byte offset.
            const double need = double(e.count) * double(e.recordBytes);
            const bool whole = need <= double(cur.remaining());
            const size_t rows = whole ? e.count : (e.recordBytes ? cur.remaining() / e.recordBytes : 0);
            const auto *rec = reinterpret_cast<const unsigned char *>(cur.position());
            const bool swap = cur.swap();
            for (size_t q = 0; q < e.props.size(); ++q) {
                if (target[q] < 0)
                    continue;
                const Property &p = e.props[q];
                const double div = colourScale(Column(target[q]), p.value);
                float *col = out.data[size_t(target[q])].data();
                for (size_t i = 0; i < rows; ++i) {
                    double v = decodeBinary(rec + i * e.recordBytes + p.offset, p.value, swap);
                    if (div != 1.0)
                        v /= div;
                    col[i] = float(v);
                }
            }
            if (!whole)
                return fail(error, "Truncated PLY data at vertex " + std::to_string(rows));
            return true;
        }
        for (size_t i = 0; i < e.count; ++i)
            for (size_t q = 0; q < e.props.size(); ++q) {
                const Property &p = e.props[q];
                if (target[q] < 0) {
                    if (!cur.skip(p))
                        return fail(error, "Truncated PLY data at vertex " + std::to_string(i));
                    continue;
                }
                double v;
                if (!cur.read(p.value, v))
                    return fail(error, "Truncated PLY data at vertex " + std::to_string(i));
                const double div = colourScale(Column(target[q]), p.value);
                out.data[size_t(target[q])][i] = float(div != 1.0 ? v / div : v);
            }
        return true;
    }
    return fail(error, "PLY file has no vertex element");
}

bool readFile(const std::string &path, std::vector<char> &bytes, std::string *error)
{
    std::ifstream in(path, std::ios::binary);
    if (!in)
        return fail(error, "Cannot open " + path);
    bytes.assign(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
    return true;
}

} // namespace

// ---------------------------------------------------------------- public

bool writeSplatPlyHost(const std::string &path, const u3dg_model &m, std::string *error, const float *shRest,
                       int shDegree)
{
    if (shRest != nullptr && (shDegree < 1 || shDegree > 3))
        return fail(error, "SH degree must be 1..3 with higher-order coefficients");
    const size_t K = shRest ? size_t((shDegree + 1) * (shDegree + 1) - 1) : 0;
    std::ofstream out(path, std::ios::binary);
    if (!out)
        return fail(error, "Cannot write " + path);
    // The 3DGS property list; normals are written as zeros (SplatPly.cpp:261-282).
    static const char *const kProps[] = {"x",      "y",       "z",       "nx",      "ny",    "nz",
                                         "f_dc_0", "f_dc_1",  "f_dc_2",  "opacity", "scale_0", "scale_1",
                                         "scale_2", "rot_0",  "rot_1",   "rot_2",   "rot_3"};
    std::string head = "ply\nformat binary_little_endian 1.0\ncomment Universal 3D Reconstruction System\n";
    head += "element vertex " + std::to_string(m.count) + "\n";
    for (int j = 0; j < 17; ++j) {
        head += std::string("property float ") + kProps[j] + "\n";
        if (j == 8) // after f_dc_2
            for (size_t r = 0; r < 3 * K; ++r)
                head += "property float f_rest_" + std::to_string(r) + "\n";
    }
    head += "end_header\n";
    out.write(head.data(), std::streamsize(head.size()));
    // Records assembled in blocks of up to 64k Gaussians and written with one call per block.
    const size_t kRec = 17 + 3 * K;
    constexpr size_t kBlock = 65536;
    std::vector<float> buf;
    for (size_t first = 0; first < m.count && out; first += kBlock) {
        const size_t n = std::min(kBlock, m.count - first);
        buf.assign(n * kRec, 0.0f);
        for (size_t j = 0; j < n; ++j) {
            const size_t i = first + j;
            float *r = &buf[j * kRec];
            std::memcpy(r, m.means + i * 3, 3 * sizeof(float));
            std::memcpy(r + 6, m.colors + i * 3, 3 * sizeof(float));
            for (size_t c = 0; c < 3; ++c) // f_rest_{c K + k} from [i][k][c]
                for (size_t k = 0; k < K; ++k)
                    r[9 + c * K + k] = shRest[(i * K + k) * 3 + c];
            float *t = r + 9 + 3 * K;
            t[0] = m.opacities[i];
            std::memcpy(t + 1, m.scales + i * 3, 3 * sizeof(float));
            std::memcpy(t + 4, m.quats + i * 4, 4 * sizeof(float));
        }
        if (!hostLittleEndian())
            for (float &v : buf) {
                unsigned char b[4];
                std::memcpy(b, &v, 4);
                std::swap(b[0], b[3]);
                std::swap(b[1], b[2]);
                std::memcpy(&v, b, 4);
            }
        out.write(reinterpret_cast<const char *>(buf.data()), std::streamsize(buf.size() * sizeof(float)));
    }
    if (!out)
        return fail(error, "Write error: " + path);
    return true;
}

bool readSplatPlyHost(const std::string &path, HostModel &model, std::string *error, bool *isSplat)
{
    std::vector<char> file;
    if (!readFile(path, file, error))
        return false;
    Header h;
    std::string why;
    if (!parseHeader(file, h, &why))
        return fail(error, why + ": " + path);
    VertexColumns v;
    if (!decodeVertices(file, h, v, error))
        return false;
    if (!v.present[X] || !v.present[Y] || !v.present[Z])
        return fail(error, "PLY vertices have no x/y/z");
    const bool splat = v.present[DC0] && v.present[OPACITY] && v.present[SCALE0] && v.present[ROT0];
    if (isSplat)
        *isSplat = splat;
    auto finite = [&](size_t i) {
        return std::isfinite(v.data[X][i]) && std::isfinite(v.data[Y][i]) && std::isfinite(v.data[Z][i]);
    };
    if (!splat) {
        // A point cloud: small opaque Gaussians around its points (SplatPly.cpp:301-321).
        std::vector<float> xyz, rgb;
        xyz.reserve(v.count * 3);
        rgb.reserve(v.count * 3);
        const bool coloured = v.present[RED];
        for (size_t i = 0; i < v.count; ++i) {
            if (!finite(i))
                continue;
            for (int c = X; c <= Z; ++c)
                xyz.push_back(v.data[size_t(c)][i]);
            for (int c = RED; c <= BLUE; ++c)
                rgb.push_back(coloured ? v.data[size_t(c)][i] : 0.8f);
        }
        const size_t n = xyz.size() / 3;
        model.resize(n);
        u3dg_model out{model.means.data(), model.scales.data(), model.quats.data(), model.opac.data(),
                       model.colors.data(), n};
        initGaussiansFromPointsHost(xyz.data(), rgb.data(), n, out);
        const float opaque = std::log(0.95f / (1.0f - 0.95f)), half = std::log(0.5f);
        std::fill(model.opac.begin(), model.opac.end(), opaque);
        for (float &s : model.scales)
            s += half;
        return true;
    }
    model.resize(v.count);
    size_t kept = 0;
    for (size_t i = 0; i < v.count; ++i) {
        if (!finite(i))
            continue;
        for (int k = 0; k < 3; ++k) {
            model.means[kept * 3 + size_t(k)] = v.data[size_t(X + k)][i];
            model.colors[kept * 3 + size_t(k)] = v.data[size_t(DC0 + k)][i];
            model.scales[kept * 3 + size_t(k)] = v.data[size_t(SCALE0 + k)][i];
        }
        for (int k = 0; k < 4; ++k)
            model.quats[kept * 4 + size_t(k)] = v.data[size_t(ROT0 + k)][i];
        model.opac[kept] = v.data[OPACITY][i];
        ++kept;
    }
    model.resize(kept);
    return true;
}

} // namespace u3dg
