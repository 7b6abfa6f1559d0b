// host_io.cpp - host-side Gaussian model I/O (binary 3DGS PLY) and the plain point-cloud
// initialisation. These run once per training run, outside the hot loop.

#include "host_io.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>

namespace u3dg {

namespace {

constexpr float kC0 = 0.28209479177387814f;

float logitHost(float p) { return std::log(p / (1.0f - p)); }

} // namespace

// The reference buckets points by a hash of their grid cell and scans the 27 neighbouring keys
// (GaussianModel.cpp:84-121). Points whose cells hash to the same key share a bucket there, and
// a bucket whose key appears twice among the 27 is scanned twice; both effects change which
// distances compete for the 3 nearest, so they are kept: here the buckets are runs of a
// key-sorted index, looked up by binary search.
int64_t initHashKey(int x, int y, int z)
{
    return (int64_t(x) * 73856093) ^ (int64_t(y) * 19349663) ^ (int64_t(z) * 83492791);
}

void buildInitGrid(const float *xyz, size_t n, InitGrid &g)
{
    float lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = std::numeric_limits<float>::max();
        hi[k] = -lo[k];
    }
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], xyz[i * 3 + k]);
            hi[k] = std::max(hi[k], xyz[i * 3 + k]);
        }
    const float ext = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-6f});
    g.cell = std::max(ext / std::cbrt(float(n)) * 2.0f, 1e-6f);
    g.cx.resize(n);
    g.cy.resize(n);
    g.cz.resize(n);
    std::vector<std::pair<int64_t, uint32_t>> bucket(n);
    for (size_t i = 0; i < n; ++i) {
        g.cx[i] = int(std::floor((xyz[i * 3] - lo[0]) / g.cell));
        g.cy[i] = int(std::floor((xyz[i * 3 + 1] - lo[1]) / g.cell));
        g.cz[i] = int(std::floor((xyz[i * 3 + 2] - lo[2]) / g.cell));
        bucket[i] = {initHashKey(g.cx[i], g.cy[i], g.cz[i]), uint32_t(i)};
    }
    std::sort(bucket.begin(), bucket.end());
    g.keys.resize(n);
    g.ids.resize(n);
    for (size_t i = 0; i < n; ++i) {
        g.keys[i] = bucket[i].first;
        g.ids[i] = bucket[i].second;
    }
}

void finishInitFromNeighbours(const float *xyz, const float *rgb, size_t n, float cell, const float *best,
                              u3dg_model &out)
{
    const float fmax = std::numeric_limits<float>::max();
    const float op = logitHost(0.1f);
    for (size_t i = 0; i < n; ++i) {
        float sum = 0;
        int cnt = 0;
        for (int k = 0; k < 3; ++k)
            if (best[i * 3 + k] < fmax) {
                sum += best[i * 3 + k];
                ++cnt;
            }
        const float meanD2 = cnt ? sum / float(cnt) : cell * cell;
        const float logScale = std::log(std::sqrt(std::max(meanD2, 1e-14f)));
        for (int k = 0; k < 3; ++k) {
            out.means[i * 3 + k] = xyz[i * 3 + k];
            out.scales[i * 3 + k] = logScale;
            const float col = rgb ? rgb[i * 3 + k] : 0.5f;
            out.colors[i * 3 + k] = (col - 0.5f) / kC0;
        }
        out.quats[i * 4] = 1.0f;
        out.quats[i * 4 + 1] = out.quats[i * 4 + 2] = out.quats[i * 4 + 3] = 0.0f;
        out.opacities[i] = op;
    }
}

void initGaussiansFromPointsHost(const float *xyz, const float *rgb, size_t n, u3dg_model &out)
{
    if (n == 0)
        return;
    InitGrid g;
    buildInitGrid(xyz, n, g);
    const float fmax = std::numeric_limits<float>::max();
    std::vector<float> best(n * 3, fmax);
    for (size_t i = 0; i < n; ++i) {
        float *b = &best[i * 3];
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    const int64_t key = initHashKey(g.cx[i] + dx, g.cy[i] + dy, g.cz[i] + dz);
                    size_t it = size_t(std::lower_bound(g.keys.begin(), g.keys.end(), key) - g.keys.begin());
                    for (; it < n && g.keys[it] == key; ++it) {
                        const size_t j = g.ids[it];
                        if (j == i)
                            continue;
                        const float ex = xyz[j * 3] - xyz[i * 3], ey = xyz[j * 3 + 1] - xyz[i * 3 + 1],
                                    ez = xyz[j * 3 + 2] - xyz[i * 3 + 2];
                        float d2 = ex * ex + ey * ey + ez * ez;
                        for (int k = 0; k < 3; ++k)
                            if (d2 < b[k])
                                std::swap(d2, b[k]);
                    }
                }
    }
    finishInitFromNeighbours(xyz, rgb, n, g.cell, best.data(), out);
}

// ------------------------------------------------------------------ PLY

namespace {

bool fail(std::string *error, const std::string &m)
{
    if (error)
        *error = m;
    return false;
}

enum class PType { I8, U8, I16, U16, I32, U32, F32, F64, Bad };

PType typeOf(const std::string &t)
{
    static const std::pair<const char *, PType> names[] = {
        {"char", PType::I8},   {"int8", PType::I8},     {"uchar", PType::U8},  {"uint8", PType::U8},
        {"short", PType::I16}, {"int16", PType::I16},   {"ushort", PType::U16}, {"uint16", PType::U16},
        {"int", PType::I32},   {"int32", PType::I32},   {"uint", PType::U32},  {"uint32", PType::U32},
        {"float", PType::F32}, {"float32", PType::F32}, {"double", PType::F64}, {"float64", PType::F64}};
    for (const auto &p : names)
        if (t == p.first)
            return p.second;
    return PType::Bad;
}

int sizeOf(PType t)
{
    switch (t) {
    case PType::I8:
    case PType::U8: return 1;
    case PType::I16:
    case PType::U16: return 2;
    case PType::I32:
    case PType::U32:
    case PType::F32: return 4;
    case PType::F64: return 8;
    default: return 0;
    }
}

struct Prop {
    std::string name;
    PType type = PType::Bad, countType = PType::Bad;
    bool list = false;
};

struct Elem {
    std::string name;
    size_t count = 0;
    std::vector<Prop> props;
};

enum class Fmt { Ascii, LE, BE };

bool littleEndianHost()
{
    const uint16_t v = 1;
    uint8_t b;
    std::memcpy(&b, &v, 1);
    return b == 1;
}

// Sequential value reader over the PLY body.
struct Body {
    const char *p, *end;
    Fmt fmt;
    bool value(PType t, double &out)
    {
        if (fmt == Fmt::Ascii) {
            while (p < end && std::isspace(static_cast<unsigned char>(*p)))
                ++p;
            const char *s = p;
            while (p < end && !std::isspace(static_cast<unsigned char>(*p)))
                ++p;
            if (p == s)
                return false;
            std::istringstream ss(std::string(s, p));
            ss.imbue(std::locale::classic());
            ss >> out;
            return !ss.fail();
        }
        const int sz = sizeOf(t);
        if (sz == 0 || end - p < sz)
            return false;
        unsigned char b[8];
        std::memcpy(b, p, size_t(sz));
        p += sz;
        if ((fmt == Fmt::LE) != littleEndianHost())
            std::reverse(b, b + sz);
        switch (t) {
        case PType::I8: { int8_t v; std::memcpy(&v, b, 1); out = v; break; }
        case PType::U8: out = b[0]; break;
        case PType::I16: { int16_t v; std::memcpy(&v, b, 2); out = v; break; }
        case PType::U16: { uint16_t v; std::memcpy(&v, b, 2); out = v; break; }
        case PType::I32: { int32_t v; std::memcpy(&v, b, 4); out = v; break; }
        case PType::U32: { uint32_t v; std::memcpy(&v, b, 4); out = v; break; }
        case PType::F32: { float v; std::memcpy(&v, b, 4); out = v; break; }
        case PType::F64: { double v; std::memcpy(&v, b, 8); out = v; break; }
        default: return false;
        }
        return true;
    }
    bool skip(const Prop &q)
    {
        double v;
        if (!q.list)
            return fmt == Fmt::Ascii ? value(q.type, v) : advance(sizeOf(q.type));
        double c;
        if (!value(q.countType, c) || c < 0)
            return false;
        for (size_t k = 0; k < size_t(c); ++k)
            if (!(fmt == Fmt::Ascii ? value(q.type, v) : advance(sizeOf(q.type))))
                return false;
        return true;
    }
    bool advance(int n)
    {
        if (end - p < n)
            return false;
        p += n;
        return true;
    }
};

// Reads the vertex table: one row of `wanted.size()` values per vertex (NaN where missing).
bool readVertices(const std::string &path, const std::vector<std::string> &wanted, std::vector<float> &rows,
                  std::vector<bool> &found, size_t &count, std::string *error)
{
    std::ifstream in(path, std::ios::binary);
    if (!in)
        return fail(error, "Cannot open " + path);
    std::vector<char> data((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    const std::string head(data.data(), std::min<size_t>(data.size(), 1 << 16));
    if (head.compare(0, 3, "ply") != 0)
        return fail(error, "Not a PLY file: " + path);
    const size_t endHeader = head.find("end_header");
    if (endHeader == std::string::npos)
        return fail(error, "PLY header has no end_header");
    const size_t bodyStart = head.find('\n', endHeader);
    if (bodyStart == std::string::npos)
        return fail(error, "Truncated PLY header");
    Fmt fmt = Fmt::Ascii;
    std::vector<Elem> elems;
    std::istringstream hs(head.substr(0, endHeader));
    std::string line;
    while (std::getline(hs, line)) {
        std::istringstream ls(line);
        std::string w;
        ls >> w;
        if (w == "format") {
            std::string f;
            ls >> f;
            if (f == "ascii")
                fmt = Fmt::Ascii;
            else if (f == "binary_little_endian")
                fmt = Fmt::LE;
            else if (f == "binary_big_endian")
                fmt = Fmt::BE;
            else
                return fail(error, "Unknown PLY format " + f);
        } else if (w == "element") {
            Elem e;
            ls >> e.name >> e.count;
            elems.push_back(e);
        } else if (w == "property" && !elems.empty()) {
            Prop q;
            std::string a, b, c;
            ls >> a >> b >> c;
            if (a == "list") {
                q.list = true;
                q.countType = typeOf(b);
                q.type = typeOf(c);
                ls >> q.name;
            } else {
                q.type = typeOf(a);
                q.name = b;
            }
            if (q.type == PType::Bad)
                return fail(error, "Unsupported PLY property: " + line);
            elems.back().props.push_back(q);
        }
    }
    Body body{data.data() + bodyStart + 1, data.data() + data.size(), fmt};
    for (const Elem &e : elems) {
        if (e.name != "vertex") {
            for (size_t i = 0; i < e.count; ++i)
                for (const Prop &q : e.props)
                    if (!body.skip(q))
                        return fail(error, "Truncated PLY data");
            continue;
        }
        std::vector<int> column(e.props.size(), -1);
        found.assign(wanted.size(), false);
        for (size_t k = 0; k < wanted.size(); ++k)
            for (size_t q = 0; q < e.props.size(); ++q)
                if (!e.props[q].list && e.props[q].name == wanted[k]) {
                    column[q] = int(k);
                    found[k] = true;
                }
        count = e.count;
        rows.assign(e.count * wanted.size(), std::nanf(""));
        for (size_t i = 0; i < e.count; ++i)
            for (size_t q = 0; q < e.props.size(); ++q) {
                if (column[q] < 0) {
                    if (!body.skip(e.props[q]))
                        return fail(error, "Truncated PLY data at vertex " + std::to_string(i));
                    continue;
                }
                double v;
                if (!body.value(e.props[q].type, v))
                    return fail(error, "Truncated PLY data at vertex " + std::to_string(i));
                const std::string &name = wanted[size_t(column[q])];
                if (name == "red" || name == "green" || name == "blue") {
                    if (e.props[q].type == PType::U8)
                        v /= 255.0;
                    else if (e.props[q].type == PType::U16)
                        v /= 65535.0;
                }
                rows[i * wanted.size() + size_t(column[q])] = float(v);
            }
        return true;
    }
    return fail(error, "PLY file has no vertex element");
}

void putFloatLE(std::ofstream &out, float v)
{
    unsigned char b[4];
    std::memcpy(b, &v, 4);
    if (!littleEndianHost())
        std::reverse(b, b + 4);
    out.write(reinterpret_cast<const char *>(b), 4);
}

} // namespace

bool writeSplatPlyHost(const std::string &path, const u3dg_model &m, std::string *error)
{
    std::ofstream out(path, std::ios::binary);
    if (!out)
        return fail(error, "Cannot write " + path);
    static const char *props[] = {"x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2", "opacity",
                                  "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"};
    out << "ply\nformat binary_little_endian 1.0\n";
    out << "comment Universal 3D Reconstruction System\n";
    out << "element vertex " << m.count << "\n";
    for (const char *p : props)
        out << "property float " << p << "\n";
    out << "end_header\n";
    for (size_t i = 0; i < m.count; ++i) {
        for (int k = 0; k < 3; ++k)
            putFloatLE(out, m.means[i * 3 + k]);
        for (int k = 0; k < 3; ++k)
            putFloatLE(out, 0.0f);
        for (int k = 0; k < 3; ++k)
            putFloatLE(out, m.colors[i * 3 + k]);
        putFloatLE(out, m.opacities[i]);
        for (int k = 0; k < 3; ++k)
            putFloatLE(out, m.scales[i * 3 + k]);
        for (int k = 0; k < 4; ++k)
            putFloatLE(out, m.quats[i * 4 + k]);
    }
    if (!out)
        return fail(error, "Write error: " + path);
    return true;
}

bool readSplatPlyHost(const std::string &path, HostModel &model, std::string *error, bool *isSplat)
{
    const std::vector<std::string> wanted = {"x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0",
                                             "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3", "red",
                                             "green", "blue"};
    std::vector<float> rows;
    std::vector<bool> found;
    size_t count = 0;
    if (!readVertices(path, wanted, rows, found, count, error))
        return false;
    if (!found[0] || !found[1] || !found[2])
        return fail(error, "PLY vertices have no x/y/z");
    const bool splat = found[3] && found[6] && found[7] && found[10];
    if (isSplat)
        *isSplat = splat;
    const size_t W = wanted.size();
    if (!splat) {
        // A plain point cloud becomes small opaque Gaussians (SplatPly.cpp:301-321).
        std::vector<float> xyz, rgb;
        for (size_t i = 0; i < count; ++i) {
            const float *r = &rows[i * W];
            if (!std::isfinite(r[0]) || !std::isfinite(r[1]) || !std::isfinite(r[2]))
                continue;
            xyz.insert(xyz.end(), {r[0], r[1], r[2]});
            if (found[14])
                rgb.insert(rgb.end(), {r[14], r[15], r[16]});
            else
                rgb.insert(rgb.end(), {0.8f, 0.8f, 0.8f});
        }
        const size_t n = xyz.size() / 3;
        model.resize(n);
        u3dg_model v{model.means.data(), model.scales.data(), model.quats.data(), model.opac.data(),
                     model.colors.data(), n};
        initGaussiansFromPointsHost(xyz.data(), rgb.data(), n, v);
        const float o = logitHost(0.95f), ls = std::log(0.5f);
        for (float &x : model.opac)
            x = o;
        for (float &s : model.scales)
            s += ls;
        return true;
    }
    model.resize(count);
    size_t out = 0;
    for (size_t i = 0; i < count; ++i) {
        const float *r = &rows[i * W];
        if (!std::isfinite(r[0]) || !std::isfinite(r[1]) || !std::isfinite(r[2]))
            continue;
        for (int k = 0; k < 3; ++k) {
            model.means[out * 3 + k] = r[k];
            model.colors[out * 3 + k] = r[3 + k];
            model.scales[out * 3 + k] = r[7 + k];
        }
        model.opac[out] = r[6];
        for (int k = 0; k < 4; ++k)
            model.quats[out * 4 + k] = r[10 + k];
        ++out;
    }
    model.resize(out);
    return true;
}

} // namespace u3dg
