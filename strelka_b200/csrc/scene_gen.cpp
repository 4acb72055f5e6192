// scene_gen.cpp — seeded synthetic scenes for the benchmark configurations.
//
// Each generator fills the host buffers the reference uploads at frame 0
// (src/render/ptrender.cpp:412-639) and builds the flattened BVH over the
// world-space triangles the way PtRender::createBvhBuffer does
// (ptrender.cpp:460-511).  World positions for the BVH are computed with the
// kernels' own operation order for mul(objectToWorld, float4(p, 1)), so every
// triangle the kernels reconstruct lies exactly inside its leaf's ancestors.
//
// Random numbers come from std::mt19937_64 with explicit conversions (the
// standard distributions are implementation-defined).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <random>
#include <unordered_map>
#include <vector>

#include "../../include/strelka_b200_scenes.h"
#include "common.h"

namespace {

struct Rng {
    std::mt19937_64 g;
    explicit Rng(uint64_t seed) : g(seed) {}
    double u01() { return (double)(g() >> 11) * (1.0 / 9007199254740992.0); }
    double uniform(double a, double b) { return a + (b - a) * u01(); }
    double normal()
    {
        double u1 = u01();
        double u2 = u01();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
    }
    void unit_vector(double v[3])
    {
        // Marsaglia (1972): uniform on the sphere
        double x1, x2, s;
        do {
            x1 = uniform(-1.0, 1.0);
            x2 = uniform(-1.0, 1.0);
            s = x1 * x1 + x2 * x2;
        } while (s >= 1.0);
        double r = 2.0 * std::sqrt(1.0 - s);
        v[0] = x1 * r;
        v[1] = x2 * r;
        v[2] = 1.0 - 2.0 * s;
    }
};

// ---------------------------------------------------------------------------
// Matrices (double; column-major like glm: M[r][c] = m[c*4 + r]).
struct M4 {
    double m[16];
};
M4 identity()
{
    M4 r{};
    r.m[0] = r.m[5] = r.m[10] = r.m[15] = 1.0;
    return r;
}
M4 mul(const M4& a, const M4& b)
{
    M4 r{};
    for (int c = 0; c < 4; ++c)
        for (int rr = 0; rr < 4; ++rr) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s += a.m[k * 4 + rr] * b.m[c * 4 + k];
            r.m[c * 4 + rr] = s;
        }
    return r;
}
M4 transpose(const M4& a)
{
    M4 r{};
    for (int c = 0; c < 4; ++c)
        for (int rr = 0; rr < 4; ++rr) r.m[c * 4 + rr] = a.m[rr * 4 + c];
    return r;
}
M4 inverse(const M4& a)
{
    // Gauss-Jordan with partial pivoting on the row-major copy
    double A[4][8];
    for (int r = 0; r < 4; ++r) {
        for (int c = 0; c < 4; ++c) {
            A[r][c] = a.m[c * 4 + r];
            A[r][c + 4] = (r == c) ? 1.0 : 0.0;
        }
    }
    for (int col = 0; col < 4; ++col) {
        int piv = col;
        for (int r = col + 1; r < 4; ++r)
            if (std::fabs(A[r][col]) > std::fabs(A[piv][col])) piv = r;
        if (piv != col)
            for (int c = 0; c < 8; ++c) std::swap(A[col][c], A[piv][c]);
        double d = A[col][col];
        for (int c = 0; c < 8; ++c) A[col][c] /= d;
        for (int r = 0; r < 4; ++r) {
            if (r == col) continue;
            double f = A[r][col];
            for (int c = 0; c < 8; ++c) A[r][c] -= f * A[col][c];
        }
    }
    M4 r{};
    for (int rr = 0; rr < 4; ++rr)
        for (int c = 0; c < 4; ++c) r.m[c * 4 + rr] = A[rr][c + 4];
    return r;
}
M4 translate(double x, double y, double z)
{
    M4 r = identity();
    r.m[12] = x;
    r.m[13] = y;
    r.m[14] = z;
    return r;
}
M4 scale(double x, double y, double z)
{
    M4 r = identity();
    r.m[0] = x;
    r.m[5] = y;
    r.m[10] = z;
    return r;
}
M4 rotate_axis(const double axis[3], double angle)
{
    double x = axis[0], y = axis[1], z = axis[2];
    double n = std::sqrt(x * x + y * y + z * z);
    x /= n;
    y /= n;
    z /= n;
    double c = std::cos(angle), s = std::sin(angle), t = 1.0 - c;
    M4 r = identity();
    // rows of the rotation matrix (Rodrigues)
    double R[3][3] = {{t * x * x + c, t * x * y - s * z, t * x * z + s * y},
                      {t * x * y + s * z, t * y * y + c, t * y * z - s * x},
                      {t * x * z - s * y, t * y * z + s * x, t * z * z + c}};
    for (int rr = 0; rr < 3; ++rr)
        for (int cc = 0; cc < 3; ++cc) r.m[cc * 4 + rr] = R[rr][cc];
    return r;
}
void to_float(const M4& a, StrelkaFloat4x4& out)
{
    for (int i = 0; i < 16; ++i) out.m[i] = (float)a.m[i];
}

// mul(M, float4(p, 1)).xyz in the kernels' operation order (no contraction)
void xform_point(const StrelkaFloat4x4& M, const float p[3], float out[3])
{
    const float* m = M.m;
    for (int i = 0; i < 3; ++i)
        out[i] = ((m[0 * 4 + i] * p[0] + m[1 * 4 + i] * p[1]) + m[2 * 4 + i] * p[2]) + m[3 * 4 + i] * 1.0f;
}

// src/scene/scene.cpp:107-113 / src/hdStrelka/RenderPass.cpp:50-56
uint32_t pack_normal(const double n[3])
{
    float x = (float)n[0], y = (float)n[1], z = (float)n[2];
    uint32_t packed = (uint32_t)((x + 1.0f) / 2.0f * 511.99999f);
    packed += (uint32_t)((y + 1.0f) / 2.0f * 511.99999f) << 10;
    packed += (uint32_t)((z + 1.0f) / 2.0f * 511.99999f) << 20;
    return packed;
}
// src/hdStrelka/RenderPass.cpp:58-64
uint32_t pack_uv(double u, double v)
{
    float fu = (float)u, fv = (float)v;
    uint32_t packed = (uint32_t)((fu + 10.0f) / 20.0f * 16383.99999f);
    packed += (uint32_t)((fv + 10.0f) / 20.0f * 16383.99999f) << 16;
    return packed;
}

// ---------------------------------------------------------------------------
// Scene assembly
struct Builder {
    std::vector<Vertex> vb;
    std::vector<uint32_t> ib;
    std::vector<InstanceConstants> inst;
    std::vector<UniformLight> lights;
    std::vector<MdlMaterial> mats;
    std::vector<uint8_t> args;
    std::vector<Mdl_resource_info> resInfos;
    std::vector<std::vector<uint8_t>> textures;
    std::vector<uint32_t> texW, texH;
    std::vector<float> env;
    uint32_t envW = 0, envH = 0;
    struct Mesh {
        uint32_t indexOffset, indexCount;
    };
    std::vector<Mesh> meshes;

    uint32_t add_mesh(const std::vector<Vertex>& v, const std::vector<uint32_t>& idx)
    {
        uint32_t base = (uint32_t)vb.size();
        Mesh m{(uint32_t)ib.size(), (uint32_t)idx.size()};
        vb.insert(vb.end(), v.begin(), v.end());
        for (uint32_t i : idx) ib.push_back(i + base);
        meshes.push_back(m);
        return (uint32_t)meshes.size() - 1;
    }
    uint32_t add_material(int fn, const float base[3], float roughness, float ior, uint32_t texResource)
    {
        StrelkaMaterialArgs a{};
        for (int i = 0; i < 3; ++i) a.base_color[i] = base[i];
        a.roughness = roughness;
        a.ior = ior;
        a.base_color_texture = texResource;
        MdlMaterial m{};
        m.arg_block_offset = (int32_t)args.size();
        m.ro_data_segment_offset = 0;
        m.functionId = fn;
        args.resize(args.size() + sizeof(a));
        memcpy(args.data() + m.arg_block_offset, &a, sizeof(a));
        mats.push_back(m);
        return (uint32_t)mats.size() - 1;
    }
    // src/render/ptrender.cpp:570-590
    uint32_t add_instance(uint32_t mesh, int32_t material, const M4& xf, int32_t lightId)
    {
        InstanceConstants ic{};
        to_float(xf, ic.objectToWorld);
        to_float(inverse(xf), ic.worldToObject);
        to_float(inverse(transpose(xf)), ic.normalMatrix);
        ic.materialId = material;
        ic.indexOffset = (int32_t)meshes[mesh].indexOffset;
        ic.indexCount = (int32_t)meshes[mesh].indexCount;
        ic.lightId = lightId;
        inst.push_back(ic);
        return (uint32_t)inst.size() - 1;
    }

    int finish(StrelkaHostScene* out)
    {
        memset(out, 0, sizeof(*out));
        // world-space triangles for the BVH (ptrender.cpp:468-506)
        std::vector<BVHInputPosition> pos;
        size_t ntri = 0;
        for (auto& ic : inst) ntri += (size_t)ic.indexCount / 3;
        pos.resize(ntri * 3);
        std::vector<size_t> first(inst.size() + 1, 0);
        for (size_t i = 0; i < inst.size(); ++i) first[i + 1] = first[i] + (size_t)inst[i].indexCount / 3;
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t ii = 0; ii < (int64_t)inst.size(); ++ii) {
            const InstanceConstants& ic = inst[ii];
            const uint32_t tc = (uint32_t)ic.indexCount / 3;
            for (uint32_t t = 0; t < tc; ++t) {
                for (int k = 0; k < 3; ++k) {
                    uint32_t vi = ib[(size_t)ic.indexOffset + t * 3 + k];
                    BVHInputPosition& p = pos[(first[ii] + t) * 3 + k];
                    xform_point(ic.objectToWorld, vb[vi].position, p.pos);
                    p.instId = (uint32_t)ii;
                    p.primId = t;
                }
            }
        }
        BVHNode* nodes = nullptr;
        uint32_t numNodes = 0;
        int rc = strelka_bvh_build(pos.data(), (uint32_t)pos.size(), &nodes, &numNodes);
        if (rc) return rc;
        out->nodes = nodes;
        out->numNodes = numNodes;
        out->numTriangles = (uint32_t)ntri;
        auto dup = [](const void* src, size_t bytes) -> void* {
            void* p = malloc(bytes ? bytes : 1);
            if (bytes) memcpy(p, src, bytes);
            return p;
        };
        out->vb = (Vertex*)dup(vb.data(), vb.size() * sizeof(Vertex));
        out->numVertices = (uint32_t)vb.size();
        out->ib = (uint32_t*)dup(ib.data(), ib.size() * 4);
        out->numIndices = (uint32_t)ib.size();
        out->instances = (InstanceConstants*)dup(inst.data(), inst.size() * sizeof(InstanceConstants));
        out->numInstances = (uint32_t)inst.size();
        std::vector<UniformLight> lcopy = lights;
        if (lcopy.empty()) lcopy.push_back(UniformLight{});
        out->lights = (UniformLight*)dup(lcopy.data(), lcopy.size() * sizeof(UniformLight));
        out->numLights = (uint32_t)lights.size();
        out->materials = (MdlMaterial*)dup(mats.data(), mats.size() * sizeof(MdlMaterial));
        out->numMaterials = (uint32_t)mats.size();
        out->argBlock = (uint8_t*)dup(args.data(), args.size());
        out->argBlockBytes = args.size();
        out->resourceInfos = (Mdl_resource_info*)dup(resInfos.data(), resInfos.size() * sizeof(Mdl_resource_info));
        out->numResourceInfos = (uint32_t)resInfos.size();
        out->numTextures = (uint32_t)textures.size();
        if (!textures.empty()) {
            out->textures = (uint8_t**)malloc(textures.size() * sizeof(uint8_t*));
            out->texWidth = (uint32_t*)malloc(textures.size() * 4);
            out->texHeight = (uint32_t*)malloc(textures.size() * 4);
            for (size_t i = 0; i < textures.size(); ++i) {
                out->textures[i] = (uint8_t*)dup(textures[i].data(), textures[i].size());
                out->texWidth[i] = texW[i];
                out->texHeight[i] = texH[i];
            }
        }
        if (!env.empty()) {
            out->envRGBA = (float*)dup(env.data(), env.size() * 4);
            out->envWidth = envW;
            out->envHeight = envH;
            out->envMarginalCdf = (float*)malloc((envH + 1) * sizeof(float));
            out->envConditionalCdf = (float*)malloc((size_t)envH * (envW + 1) * sizeof(float));
            strelka_envmap_build_cdf_host(out->envRGBA, envW, envH, out->envMarginalCdf, out->envConditionalCdf,
                                          &out->envIntegral);
        }
        return STRELKA_OK;
    }
};

// ---------------------------------------------------------------------------
// Camera: src/scene/camera.cpp:61-131 (reverse-Z perspective, near/far swapped)
void set_camera(PathTracerParam& p, uint32_t W, uint32_t H, const double eye[3], const double target[3], double fovDeg)
{
    memset(&p, 0, sizeof(p));
    const float fov = (float)fovDeg;
    const float aspect = (float)W / (float)H;
    const float zfar = 1000.0f, znear = 0.01f;
    const float n = zfar, f = znear;  // swapped for reverse Z (camera.cpp:127)
    float focal_length = 1.0f / std::tan(fov * (float)(M_PI / 180.0) / 2.0f);
    float x = focal_length / aspect;
    float y = -focal_length;
    float A = n / (f - n);
    float B = f * A;
    // projection rows (x,0,0,0), (0,y,0,0), (0,0,A,B), (0,0,-1,0)
    StrelkaFloat4x4 P{}, IP{};
    P.m[0 * 4 + 0] = x;
    P.m[1 * 4 + 1] = y;
    P.m[2 * 4 + 2] = A;
    P.m[3 * 4 + 2] = B;
    P.m[2 * 4 + 3] = -1.0f;
    // inverse rows (1/x,0,0,0), (0,1/y,0,0), (0,0,0,-1), (0,0,1/B,A/B)
    IP.m[0 * 4 + 0] = 1 / x;
    IP.m[1 * 4 + 1] = 1 / y;
    IP.m[3 * 4 + 2] = -1.0f;
    IP.m[2 * 4 + 3] = 1 / B;
    IP.m[3 * 4 + 3] = A / B;
    // view = lookAt (right-handed, camera looks down -z)
    double fwd[3] = {target[0] - eye[0], target[1] - eye[1], target[2] - eye[2]};
    double fl = std::sqrt(fwd[0] * fwd[0] + fwd[1] * fwd[1] + fwd[2] * fwd[2]);
    for (double& c : fwd) c /= fl;
    double up[3] = {0.0, 1.0, 0.0};
    double right[3] = {fwd[1] * up[2] - fwd[2] * up[1], fwd[2] * up[0] - fwd[0] * up[2], fwd[0] * up[1] - fwd[1] * up[0]};
    double rl = std::sqrt(right[0] * right[0] + right[1] * right[1] + right[2] * right[2]);
    for (double& c : right) c /= rl;
    double u2[3] = {right[1] * fwd[2] - right[2] * fwd[1], right[2] * fwd[0] - right[0] * fwd[2],
                    right[0] * fwd[1] - right[1] * fwd[0]};
    M4 view = identity();
    for (int c = 0; c < 3; ++c) {
        view.m[c * 4 + 0] = right[c];
        view.m[c * 4 + 1] = u2[c];
        view.m[c * 4 + 2] = -fwd[c];
    }
    view.m[12] = -(right[0] * eye[0] + right[1] * eye[1] + right[2] * eye[2]);
    view.m[13] = -(u2[0] * eye[0] + u2[1] * eye[1] + u2[2] * eye[2]);
    view.m[14] = (fwd[0] * eye[0] + fwd[1] * eye[1] + fwd[2] * eye[2]);
    // src/render/ptrender.cpp:755-774
    to_float(inverse(view), p.viewToWorld);
    p.clipToView = IP;
    p.viewToClip = P;
    to_float(view, p.worldToView);
    p.camPos.x = (float)eye[0];
    p.camPos.y = (float)eye[1];
    p.camPos.z = (float)eye[2];
    p.camPos.w = 1.0f;
    p.dimension[0] = (int32_t)W;
    p.dimension[1] = (int32_t)H;
    p.invDimension[0] = 1.0f / (float)W;
    p.invDimension[1] = 1.0f / (float)H;
    p.spp = 1;
    p.maxDepth = 4;
}

// ---------------------------------------------------------------------------
// Icosphere: the icosahedron and midpoint subdivision of scene.cpp:142-316.
void icosahedron(std::vector<std::array<double, 3>>& v, std::vector<uint32_t>& f)
{
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    const double raw[12][3] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                               {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    v.clear();
    for (auto& r : raw) {
        double n = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        v.push_back({r[0] / n, r[1] / n, r[2] / n});
    }
    const uint32_t faces[20][3] = {{0, 11, 5}, {0, 5, 1},  {0, 1, 7},   {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
                                   {11, 10, 2}, {10, 7, 6}, {7, 1, 8},  {3, 9, 4},  {3, 4, 2},   {3, 2, 6}, {3, 6, 8},
                                   {3, 8, 9},  {4, 9, 5},  {2, 4, 11}, {6, 2, 10}, {8, 6, 7},   {9, 8, 1}};
    f.clear();
    for (auto& fc : faces) f.insert(f.end(), {fc[0], fc[1], fc[2]});
}

void subdivide(std::vector<std::array<double, 3>>& v, std::vector<uint32_t>& f)
{
    std::map<std::pair<uint32_t, uint32_t>, uint32_t> lookup;
    auto mid = [&](uint32_t a, uint32_t b) {
        auto key = a < b ? std::make_pair(a, b) : std::make_pair(b, a);
        auto it = lookup.find(key);
        if (it != lookup.end()) return it->second;
        std::array<double, 3> p = {(v[a][0] + v[b][0]) / 2, (v[a][1] + v[b][1]) / 2, (v[a][2] + v[b][2]) / 2};
        double n = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        for (double& c : p) c /= n;
        v.push_back(p);
        uint32_t id = (uint32_t)v.size() - 1;
        lookup[key] = id;
        return id;
    };
    std::vector<uint32_t> out;
    for (size_t i = 0; i < f.size(); i += 3) {
        uint32_t m0 = mid(f[i], f[i + 1]), m1 = mid(f[i + 1], f[i + 2]), m2 = mid(f[i + 2], f[i]);
        out.insert(out.end(), {f[i], m0, m2, f[i + 1], m1, m0, f[i + 2], m2, m1, m0, m1, m2});
    }
    f.swap(out);
}

// Geodesic sphere of frequency n: every icosahedron face split into n^2
// triangles, vertices shared across faces.
void geodesic(uint32_t n, std::vector<std::array<double, 3>>& v, std::vector<uint32_t>& f)
{
    std::vector<std::array<double, 3>> ico;
    std::vector<uint32_t> faces;
    icosahedron(ico, faces);
    std::unordered_map<uint64_t, uint32_t> ids;
    v.clear();
    f.clear();
    auto vid = [&](uint32_t a, uint32_t b, uint32_t c, uint32_t i, uint32_t j) {
        // barycentric weights (n-i-j, i, j) on corners a, b, c
        uint32_t w[3] = {n - i - j, i, j};
        uint32_t cv[3] = {a, b, c};
        std::pair<uint32_t, uint32_t> pr[3];
        int k = 0;
        for (int q = 0; q < 3; ++q)
            if (w[q]) pr[k++] = {cv[q], w[q]};
        std::sort(pr, pr + k);
        uint64_t key = (uint64_t)k;
        for (int q = 0; q < k; ++q) key = key * 4096 + pr[q].first * 256 + pr[q].second;
        auto it = ids.find(key);
        if (it != ids.end()) return it->second;
        std::array<double, 3> p = {0, 0, 0};
        for (int q = 0; q < 3; ++q)
            for (int d = 0; d < 3; ++d) p[d] += (double)w[q] * ico[cv[q]][d];
        double len = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        for (double& c : p) c /= len;
        v.push_back(p);
        uint32_t id = (uint32_t)v.size() - 1;
        ids[key] = id;
        return id;
    };
    for (size_t fi = 0; fi < faces.size(); fi += 3) {
        uint32_t a = faces[fi], b = faces[fi + 1], c = faces[fi + 2];
        for (uint32_t j = 0; j < n; ++j) {
            for (uint32_t i = 0; i + j < n; ++i) {
                uint32_t p0 = vid(a, b, c, i, j), p1 = vid(a, b, c, i + 1, j), p2 = vid(a, b, c, i, j + 1);
                f.insert(f.end(), {p0, p1, p2});
                if (i + j + 1 < n) {
                    uint32_t p3 = vid(a, b, c, i + 1, j + 1);
                    f.insert(f.end(), {p1, p3, p2});
                }
            }
        }
    }
}

// Improved noise (Perlin 2002) with a seeded permutation.
struct Perlin {
    int p[512];
    explicit Perlin(uint64_t seed)
    {
        int perm[256];
        for (int i = 0; i < 256; ++i) perm[i] = i;
        Rng r(seed);
        for (int i = 255; i > 0; --i) {
            int j = (int)(r.u01() * (i + 1));
            std::swap(perm[i], perm[j]);
        }
        for (int i = 0; i < 512; ++i) p[i] = perm[i & 255];
    }
    static double fade(double t) { return t * t * t * (t * (t * 6 - 15) + 10); }
    static double lerp(double t, double a, double b) { return a + t * (b - a); }
    static double grad(int h, double x, double y, double z)
    {
        h &= 15;
        double u = h < 8 ? x : y;
        double v = h < 4 ? y : (h == 12 || h == 14 ? x : z);
        return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
    }
    double noise(double x, double y, double z) const
    {
        int X = (int)std::floor(x) & 255, Y = (int)std::floor(y) & 255, Z = (int)std::floor(z) & 255;
        x -= std::floor(x);
        y -= std::floor(y);
        z -= std::floor(z);
        double u = fade(x), v = fade(y), w = fade(z);
        int A = p[X] + Y, AA = p[A] + Z, AB = p[A + 1] + Z, B = p[X + 1] + Y, BA = p[B] + Z, BB = p[B + 1] + Z;
        return lerp(w,
                    lerp(v, lerp(u, grad(p[AA], x, y, z), grad(p[BA], x - 1, y, z)),
                         lerp(u, grad(p[AB], x, y - 1, z), grad(p[BB], x - 1, y - 1, z))),
                    lerp(v, lerp(u, grad(p[AA + 1], x, y, z - 1), grad(p[BA + 1], x - 1, y, z - 1)),
                         lerp(u, grad(p[AB + 1], x, y - 1, z - 1), grad(p[BB + 1], x - 1, y - 1, z - 1))));
    }
};

Vertex make_vertex(const double p[3], const double n[3], double u, double v)
{
    Vertex vx{};
    for (int i = 0; i < 3; ++i) vx.position[i] = (float)p[i];
    vx.normal = pack_normal(n);
    vx.tangent = 0;
    vx.uv = pack_uv(u, v);
    return vx;
}

// quad (a,b,c,d) counter-clockwise seen from the side its normal points to
void add_quad(std::vector<Vertex>& v, std::vector<uint32_t>& idx, const double a[3], const double b[3], const double c[3],
              const double d[3], const double n[3])
{
    uint32_t base = (uint32_t)v.size();
    v.push_back(make_vertex(a, n, 0, 0));
    v.push_back(make_vertex(b, n, 1, 0));
    v.push_back(make_vertex(c, n, 1, 1));
    v.push_back(make_vertex(d, n, 0, 1));
    idx.insert(idx.end(), {base, base + 1, base + 2, base + 2, base + 3, base});
}

}  // namespace

// ---------------------------------------------------------------------------
extern "C" int strelka_envmap_build_cdf_host(const float* rgba, uint32_t W, uint32_t H, float* marginal, float* conditional,
                                             float* integral)
{
    if (!rgba || !marginal || !conditional || W == 0 || H == 0) return sb::fail(STRELKA_ERR_INVALID_ARGUMENT, "bad env map");
    std::vector<double> rowSum(H, 0.0);
    for (uint32_t y = 0; y < H; ++y) {
        double sinT = std::sin(((double)y + 0.5) / H * M_PI);
        float* c = conditional + (size_t)y * (W + 1);
        double acc = 0.0;
        std::vector<double> cum(W + 1, 0.0);
        for (uint32_t x = 0; x < W; ++x) {
            const float* p = rgba + 4 * ((size_t)y * W + x);
            double lum = 0.2126 * p[0] + 0.7152 * p[1] + 0.0722 * p[2];
            acc += std::max(lum, 0.0) * sinT;
            cum[x + 1] = acc;
        }
        rowSum[y] = acc;
        for (uint32_t x = 0; x <= W; ++x) c[x] = acc > 0 ? (float)(cum[x] / acc) : (float)x / (float)W;
        c[W] = 1.0f;
    }
    double tot = 0.0;
    std::vector<double> cum(H + 1, 0.0);
    for (uint32_t y = 0; y < H; ++y) {
        tot += rowSum[y];
        cum[y + 1] = tot;
    }
    for (uint32_t y = 0; y <= H; ++y) marginal[y] = tot > 0 ? (float)(cum[y] / tot) : (float)y / (float)H;
    marginal[H] = 1.0f;
    if (integral) *integral = (float)(tot * (2.0 * M_PI / W) * (M_PI / H));
    return STRELKA_OK;
}

extern "C" int strelka_scene_cornell(const StrelkaCornellConfig* cfg, StrelkaHostScene* out)
{
    if (!cfg || !out || cfg->width == 0 || cfg->height == 0) return sb::fail(STRELKA_ERR_INVALID_ARGUMENT, "bad config");
    Builder b;
    // materials: Lambert albedos fixed per object in [0.2, 0.8]
    const float white[3] = {0.75f, 0.75f, 0.75f}, red[3] = {0.75f, 0.2f, 0.2f}, green[3] = {0.2f, 0.75f, 0.2f};
    const float s0[3] = {0.6f, 0.6f, 0.3f}, s1[3] = {0.3f, 0.5f, 0.7f};
    uint32_t mWhite = b.add_material(STRELKA_FN_LAMBERT, white, 1.0f, 1.5f, 0);
    uint32_t mRed = b.add_material(STRELKA_FN_LAMBERT, red, 1.0f, 1.5f, 0);
    uint32_t mGreen = b.add_material(STRELKA_FN_LAMBERT, green, 1.0f, 1.5f, 0);
    uint32_t mS0 = b.add_material(STRELKA_FN_LAMBERT, s0, 1.0f, 1.5f, 0);
    uint32_t mS1 = b.add_material(STRELKA_FN_LAMBERT, s1, 1.0f, 1.5f, 0);
    // walls of the unit box, inward normals; the front (z = 1) is open
    struct Wall {
        double a[3], b[3], c[3], d[3], n[3];
        uint32_t mat;
    } walls[5] = {
        {{0, 0, 1}, {1, 0, 1}, {1, 0, 0}, {0, 0, 0}, {0, 1, 0}, mWhite},     // floor
        {{0, 1, 0}, {1, 1, 0}, {1, 1, 1}, {0, 1, 1}, {0, -1, 0}, mWhite},    // ceiling
        {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, mWhite},     // back
        {{0, 0, 1}, {0, 0, 0}, {0, 1, 0}, {0, 1, 1}, {1, 0, 0}, mRed},       // left
        {{1, 0, 0}, {1, 0, 1}, {1, 1, 1}, {1, 1, 0}, {-1, 0, 0}, mGreen},    // right
    };
    for (auto& w : walls) {
        std::vector<Vertex> v;
        std::vector<uint32_t> idx;
        add_quad(v, idx, w.a, w.b, w.c, w.d, w.n);
        uint32_t mesh = b.add_mesh(v, idx);
        b.add_instance(mesh, (int32_t)w.mat, identity(), -1);
    }
    // icospheres (outward normals), instanced with scale + translation
    {
        std::vector<std::array<double, 3>> pv;
        std::vector<uint32_t> f;
        icosahedron(pv, f);
        for (uint32_t i = 0; i < cfg->sphereLevels; ++i) subdivide(pv, f);
        std::vector<Vertex> v;
        for (auto& p : pv) {
            double u = 0.5 + std::atan2(p[0], -p[2]) / (2 * M_PI), vv = std::acos(std::max(-1.0, std::min(1.0, p[1]))) / M_PI;
            v.push_back(make_vertex(p.data(), p.data(), u, vv));
        }
        uint32_t mesh = b.add_mesh(v, f);
        b.add_instance(mesh, (int32_t)mS0, mul(translate(0.3, 0.2, 0.35), scale(0.2, 0.2, 0.2)), -1);
        b.add_instance(mesh, (int32_t)mS1, mul(translate(0.7, 0.18, 0.6), scale(0.18, 0.18, 0.18)), -1);
    }
    // rect light (scene.cpp:418-461, 463-483): local quad in z = 0 emitting
    // along local -z; local z maps to world +y so it faces down
    {
        const double side = cfg->lightSide;
        M4 rot = identity();
        // columns: local x -> world x, local y -> world -z, local z -> world y
        rot.m[0] = 1; rot.m[1] = 0; rot.m[2] = 0;
        rot.m[4] = 0; rot.m[5] = 0; rot.m[6] = -1;
        rot.m[8] = 0; rot.m[9] = 1; rot.m[10] = 0;
        M4 xf = mul(mul(translate(0.5, 0.998, 0.5), rot), scale(side, side, 1.0));
        UniformLight L{};
        const double corners[4][2] = {{0.5, 0.5}, {-0.5, 0.5}, {-0.5, -0.5}, {0.5, -0.5}};
        for (int k = 0; k < 4; ++k) {
            double p[4] = {corners[k][0], corners[k][1], 0.0, 1.0}, r[4] = {0, 0, 0, 0};
            for (int i = 0; i < 4; ++i)
                for (int j = 0; j < 4; ++j) r[i] += xf.m[j * 4 + i] * p[j];
            L.points[k].x = (float)r[0];
            L.points[k].y = (float)r[1];
            L.points[k].z = (float)r[2];
            L.points[k].w = (float)r[3];
        }
        L.color.x = L.color.y = L.color.z = cfg->lightRadiance;
        L.color.w = cfg->lightRadiance;
        L.type = 0;
        b.lights.push_back(L);
        // emitter mesh, scene.cpp:115-140
        std::vector<Vertex> v;
        const double n[3] = {1.0, 0.0, 0.0};
        for (int k = 0; k < 4; ++k) {
            double p[3] = {corners[k][0], corners[k][1], 0.0};
            v.push_back(make_vertex(p, n, 0, 0));
        }
        std::vector<uint32_t> idx = {0, 1, 2, 2, 3, 0};
        uint32_t mesh = b.add_mesh(v, idx);
        b.add_instance(mesh, -1, xf, 0);
    }
    // disc light (scene.cpp:318-361 mesh: a 16-triangle fan of the unit disc
    // in local z = 0; scene.cpp:480-495 record): its transform carries the
    // radius as a scale, so, as in the reference, the record's axes and
    // normal have length r and points[0].x scales the sample by r again
    if (cfg->extraLights & 1u) {
        const double r = 0.12, radiance = 10.0;
        M4 rot = identity();
        // local z -> world -y (facing down), local x -> world x, local y -> world z
        rot.m[0] = 1; rot.m[1] = 0; rot.m[2] = 0;
        rot.m[4] = 0; rot.m[5] = 0; rot.m[6] = 1;
        rot.m[8] = 0; rot.m[9] = -1; rot.m[10] = 0;
        M4 xf = mul(mul(translate(0.52, 0.93, 0.47), rot), scale(r, r, r));
        auto apply = [&](const double p[4], float out[4]) {
            for (int i = 0; i < 4; ++i) {
                double acc = 0;
                for (int j = 0; j < 4; ++j) acc += xf.m[j * 4 + i] * p[j];
                out[i] = (float)acc;
            }
        };
        UniformLight L{};
        L.points[0].x = (float)r;
        const double o[4] = {0, 0, 0, 1}, ex[4] = {1, 0, 0, 0}, ey[4] = {0, 1, 0, 0}, ez[4] = {0, 0, 1, 0};
        apply(o, &L.points[1].x);
        apply(ex, &L.points[2].x);
        apply(ey, &L.points[3].x);
        apply(ez, &L.normal.x);
        const float c = (float)(radiance);
        L.color.x = L.color.y = L.color.z = c;
        L.color.w = c;
        L.type = 1;
        const int32_t lightId = (int32_t)b.lights.size();
        b.lights.push_back(L);
        std::vector<Vertex> v;
        std::vector<uint32_t> idx;
        const double n[3] = {0.0, 0.0, 1.0};
        const double centre[3] = {0, 0, 0}, first[3] = {1, 0, 0};
        v.push_back(make_vertex(centre, n, 0, 0));
        v.push_back(make_vertex(first, n, 0, 0));
        const double step = 2.0 * M_PI / 16;
        double angle = 0;
        for (int i = 0; i < 16; ++i) {
            idx.push_back(0);
            idx.push_back((uint32_t)v.size() - 1);
            angle += step;
            const double p[3] = {std::cos(angle), std::sin(angle), 0.0};
            v.push_back(make_vertex(p, n, 0, 0));
            idx.push_back((uint32_t)v.size() - 1);
        }
        uint32_t mesh = b.add_mesh(v, idx);
        b.add_instance(mesh, -1, xf, lightId);
    }
    // sphere light (scene.cpp:210-316 mesh: an icosphere subdivided 3 times;
    // scene.cpp:497-508 record: radius and centre)
    if (cfg->extraLights & 2u) {
        const double r = 0.08, radiance = 20.0;
        M4 xf = mul(translate(0.62, 0.55, 0.62), scale(r, r, r));
        UniformLight L{};
        L.points[0].x = (float)r;
        L.points[1].x = 0.62f;
        L.points[1].y = 0.55f;
        L.points[1].z = 0.62f;
        L.points[1].w = 1.0f;
        const float c = (float)radiance;
        L.color.x = L.color.y = L.color.z = c;
        L.color.w = c;
        L.type = 2;
        const int32_t lightId = (int32_t)b.lights.size();
        b.lights.push_back(L);
        std::vector<std::array<double, 3>> pv;
        std::vector<uint32_t> f;
        icosahedron(pv, f);
        for (int i = 0; i < 3; ++i) subdivide(pv, f);
        std::vector<Vertex> v;
        for (auto& p : pv) v.push_back(make_vertex(p.data(), p.data(), 0, 0));
        uint32_t mesh = b.add_mesh(v, f);
        b.add_instance(mesh, -1, xf, lightId);
    }
    int rc = b.finish(out);
    if (rc) return rc;
    const double eye[3] = {0.5, 0.5, 2.35}, target[3] = {0.5, 0.5, 0.0};
    set_camera(out->camera, cfg->width, cfg->height, eye, target, 40.0);
    out->camera.numLights = out->numLights;
    out->camera.maxDepth = cfg->maxDepth;
    out->camera.spp = (int32_t)(cfg->spp ? cfg->spp : 1);
    return STRELKA_OK;
}

extern "C" int strelka_scene_soup(uint32_t numTris, uint64_t seed, StrelkaHostScene* out)
{
    if (!out || numTris == 0) return sb::fail(STRELKA_ERR_INVALID_ARGUMENT, "bad arguments");
    Builder b;
    const float albedo[3] = {0.5f, 0.5f, 0.5f};
    uint32_t mat = b.add_material(STRELKA_FN_LAMBERT, albedo, 1.0f, 1.5f, 0);
    std::vector<Vertex> v(3 * (size_t)numTris);
    std::vector<uint32_t> idx(3 * (size_t)numTris);
    Rng r(seed);
    const double mu = std::log(0.003), sigma = 0.5;
    for (uint32_t t = 0; t < numTris; ++t) {
        double c[3] = {r.u01(), r.u01(), r.u01()};
        double p[3][3];
        for (int k = 0; k < 3; ++k) {
            double d[3];
            r.unit_vector(d);
            double len = std::exp(mu + sigma * r.normal());
            for (int a = 0; a < 3; ++a) p[k][a] = c[a] + d[a] * len;
        }
        double e0[3], e1[3], n[3];
        for (int a = 0; a < 3; ++a) {
            e0[a] = p[1][a] - p[0][a];
            e1[a] = p[2][a] - p[0][a];
        }
        n[0] = e0[1] * e1[2] - e0[2] * e1[1];
        n[1] = e0[2] * e1[0] - e0[0] * e1[2];
        n[2] = e0[0] * e1[1] - e0[1] * e1[0];
        double nl = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        for (double& q : n) q = nl > 0 ? q / nl : 0.0;
        for (int k = 0; k < 3; ++k) {
            v[3 * (size_t)t + k] = make_vertex(p[k], n, 0, 0);
            idx[3 * (size_t)t + k] = 3 * t + k;
        }
    }
    uint32_t mesh = b.add_mesh(v, idx);
    b.add_instance(mesh, (int32_t)mat, identity(), -1);
    int rc = b.finish(out);
    if (rc) return rc;
    const double eye[3] = {0.5, 0.5, 3.0}, target[3] = {0.5, 0.5, 0.5};
    set_camera(out->camera, 512, 512, eye, target, 40.0);
    out->camera.numLights = 0;
    return STRELKA_OK;
}

extern "C" int strelka_rays_soup(uint32_t numRays, uint64_t seed, int shadow, Ray* out)
{
    if (!out && numRays) return sb::fail(STRELKA_ERR_INVALID_ARGUMENT, "out is NULL");
    Rng r(seed);
    for (uint32_t i = 0; i < numRays; ++i) {
        double o[3] = {r.uniform(-0.5, 1.5), r.uniform(-0.5, 1.5), r.uniform(-0.5, 1.5)};
        double d[3];
        r.unit_vector(d);
        double tmax = shadow ? r.uniform(0.1, 2.0) : 1e9;
        out[i].o.x = (float)o[0];
        out[i].o.y = (float)o[1];
        out[i].o.z = (float)o[2];
        out[i].o.w = (float)tmax;
        out[i].d.x = (float)d[0];
        out[i].d.y = (float)d[1];
        out[i].d.z = (float)d[2];
        out[i].d.w = 0.0f;
    }
    return STRELKA_OK;
}

extern "C" int strelka_scene_large(const StrelkaLargeConfig* cfg, StrelkaHostScene* out)
{
    if (!cfg || !out || cfg->width == 0 || cfg->height == 0 || cfg->frequency == 0 || cfg->instances == 0)
        return sb::fail(STRELKA_ERR_INVALID_ARGUMENT, "bad config");
    Builder b;
    Rng r(cfg->seed);
    // procedural noise textures (value-noise fBm, RGBA8 sRGB)
    const uint32_t T = cfg->texSize ? cfg->texSize : 2048;
    for (uint32_t t = 0; t < cfg->numTextures; ++t) {
        std::vector<uint8_t> img((size_t)T * T * 4);
        Perlin pn(cfg->seed * 7919 + t + 1);
        double base[3] = {r.uniform(0.2, 0.9), r.uniform(0.2, 0.9), r.uniform(0.2, 0.9)};
        double alt[3] = {r.uniform(0.05, 0.6), r.uniform(0.05, 0.6), r.uniform(0.05, 0.6)};
        double freq = r.uniform(4.0, 16.0);
#pragma omp parallel for schedule(static)
        for (int64_t y = 0; y < (int64_t)T; ++y) {
            for (uint32_t x = 0; x < T; ++x) {
                // tileable: sample noise on a torus
                double a = 2 * M_PI * x / T, bb = 2 * M_PI * y / T;
                double px = std::cos(a) * freq / (2 * M_PI), py = std::sin(a) * freq / (2 * M_PI);
                double pz = std::cos(bb) * freq / (2 * M_PI), pw = std::sin(bb) * freq / (2 * M_PI);
                double nsum = 0.0, amp = 0.5, f = 1.0;
                for (int o = 0; o < 4; ++o) {
                    nsum += amp * pn.noise(px * f + pz * 0.37 * f, py * f + pw * f, pz * f - py * 0.21 * f);
                    amp *= 0.5;
                    f *= 2.0;
                }
                double k = std::min(1.0, std::max(0.0, 0.5 + nsum));
                uint8_t* o8 = &img[4 * ((size_t)y * T + x)];
                for (int c = 0; c < 3; ++c) {
                    double lin = base[c] * (1 - k) + alt[c] * k;
                    double s = lin <= 0.0031308 ? lin * 12.92 : 1.055 * std::pow(lin, 1 / 2.4) - 0.055;
                    o8[c] = (uint8_t)std::lround(std::min(1.0, std::max(0.0, s)) * 255.0);
                }
                o8[3] = 255;
            }
        }
        b.textures.push_back(std::move(img));
        b.texW.push_back(T);
        b.texH.push_back(T);
        Mdl_resource_info ri{};
        ri.gpu_resource_array_start = t;
        b.resInfos.push_back(ri);
    }
    // displaced geodesic sphere, shared by every instance
    uint32_t sphereMesh;
    {
        std::vector<std::array<double, 3>> pv;
        std::vector<uint32_t> f;
        geodesic(cfg->frequency, pv, f);
        Perlin pn(cfg->seed ^ 0x9e3779b97f4a7c15ull);
        std::vector<std::array<double, 3>> disp(pv.size());
        for (size_t i = 0; i < pv.size(); ++i) {
            double h = pn.noise(pv[i][0] * 4.0 + 11.5, pv[i][1] * 4.0 + 3.25, pv[i][2] * 4.0 + 7.75);
            double rad = 1.0 + 0.05 * h;
            for (int a = 0; a < 3; ++a) disp[i][a] = pv[i][a] * rad;
        }
        std::vector<std::array<double, 3>> nrm(pv.size(), {0, 0, 0});
        for (size_t i = 0; i < f.size(); i += 3) {
            auto& a = disp[f[i]];
            auto& bq = disp[f[i + 1]];
            auto& c = disp[f[i + 2]];
            double e0[3] = {bq[0] - a[0], bq[1] - a[1], bq[2] - a[2]}, e1[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
            double n[3] = {e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0]};
            for (int k = 0; k < 3; ++k)
                for (int d = 0; d < 3; ++d) nrm[f[i + k]][d] += n[d];
        }
        std::vector<Vertex> v(pv.size());
        for (size_t i = 0; i < pv.size(); ++i) {
            double l = std::sqrt(nrm[i][0] * nrm[i][0] + nrm[i][1] * nrm[i][1] + nrm[i][2] * nrm[i][2]);
            double n[3] = {nrm[i][0] / l, nrm[i][1] / l, nrm[i][2] / l};
            double u = 0.5 + std::atan2(pv[i][0], -pv[i][2]) / (2 * M_PI);
            double vv = std::acos(std::max(-1.0, std::min(1.0, pv[i][1]))) / M_PI;
            v[i] = make_vertex(disp[i].data(), n, u * 4.0, vv * 2.0);
        }
        sphereMesh = b.add_mesh(v, f);
    }
    // ground quad
    uint32_t groundMesh;
    {
        std::vector<Vertex> v;
        std::vector<uint32_t> idx;
        const double a[3] = {-40, 0, 40}, bq[3] = {40, 0, 40}, c[3] = {40, 0, -40}, d[3] = {-40, 0, -40}, n[3] = {0, 1, 0};
        add_quad(v, idx, a, bq, c, d, n);
        groundMesh = b.add_mesh(v, idx);
    }
    const float grey[3] = {0.5f, 0.5f, 0.5f};
    uint32_t groundMat = b.add_material(STRELKA_FN_LAMBERT, grey, 1.0f, 1.5f, cfg->numTextures ? 1u : 0u);
    b.add_instance(groundMesh, (int32_t)groundMat, identity(), -1);
    // instances on a jittered grid, random rotation, scale 0.5-2
    const uint32_t N = cfg->instances;
    const uint32_t side = (uint32_t)std::ceil(std::sqrt((double)N));
    const double spacing = 4.5;
    for (uint32_t i = 0; i < N; ++i) {
        double s = r.uniform(0.5, 2.0);
        double gx = (double)(i % side) - (side - 1) * 0.5, gz = (double)(i / side) - (side - 1) * 0.5;
        double tx = gx * spacing + r.uniform(-0.8, 0.8), tz = gz * spacing + r.uniform(-0.8, 0.8);
        double ty = s * 1.05 + r.uniform(0.0, 1.5);
        double axis[3];
        r.unit_vector(axis);
        double ang = r.uniform(0.0, 2 * M_PI);
        M4 xf = mul(mul(translate(tx, ty, tz), rotate_axis(axis, ang)), scale(s, s, s));
        double pick = r.u01();
        float col[3] = {(float)r.uniform(0.2, 0.9), (float)r.uniform(0.2, 0.9), (float)r.uniform(0.2, 0.9)};
        float rough = (float)r.uniform(0.05, 1.0);
        uint32_t tex = (cfg->numTextures && r.u01() < 0.5) ? 1u + (uint32_t)(r.u01() * cfg->numTextures) % cfg->numTextures : 0u;
        int fn = pick < 0.5 ? STRELKA_FN_LAMBERT : (pick < 0.8 ? STRELKA_FN_GGX_CONDUCTOR : STRELKA_FN_GGX_DIELECTRIC);
        if (fn == STRELKA_FN_GGX_DIELECTRIC) tex = 0;
        float ior = (float)r.uniform(1.3, 1.7);
        uint32_t m = b.add_material(fn, col, rough, ior, tex);
        b.add_instance(sphereMesh, (int32_t)m, xf, -1);
    }
    // environment: sky gradient + one hot sun lobe
    {
        const uint32_t W = cfg->envWidth ? cfg->envWidth : 1024, H = cfg->envHeight ? cfg->envHeight : 512;
        b.env.resize((size_t)W * H * 4);
        b.envW = W;
        b.envH = H;
        const double sunTheta = 0.75, sunPhi = 0.9;
        const double sd[3] = {std::sin(sunTheta) * std::sin(sunPhi), std::cos(sunTheta), -std::sin(sunTheta) * std::cos(sunPhi)};
        for (uint32_t y = 0; y < H; ++y) {
            double theta = ((double)y + 0.5) / H * M_PI;
            for (uint32_t x = 0; x < W; ++x) {
                double phi = (((double)x + 0.5) / W - 0.5) * 2 * M_PI;
                double d[3] = {std::sin(theta) * std::sin(phi), std::cos(theta), -std::sin(theta) * std::cos(phi)};
                double up = std::max(0.0, d[1]);
                double sky[3] = {0.35 + 0.25 * up, 0.45 + 0.3 * up, 0.6 + 0.4 * up};
                if (d[1] < 0) {
                    sky[0] = sky[1] = sky[2] = 0.15;
                }
                double cosg = d[0] * sd[0] + d[1] * sd[1] + d[2] * sd[2];
                double lobe = std::exp((cosg - 1.0) * 4000.0) * 2.0e4;
                float* p = &b.env[4 * ((size_t)y * W + x)];
                p[0] = (float)(sky[0] + lobe * 1.0);
                p[1] = (float)(sky[1] + lobe * 0.95);
                p[2] = (float)(sky[2] + lobe * 0.85);
                p[3] = 1.0f;
            }
        }
    }
    int rc = b.finish(out);
    if (rc) return rc;
    const double eye[3] = {0.0, 9.0, 30.0}, target[3] = {0.0, 1.5, 0.0};
    set_camera(out->camera, cfg->width, cfg->height, eye, target, 40.0);
    out->camera.numLights = 0;
    out->camera.maxDepth = cfg->maxDepth;
    out->camera.spp = (int32_t)(cfg->spp ? cfg->spp : 1);
    return STRELKA_OK;
}

extern "C" int strelka_camera_lookat(PathTracerParam* p, uint32_t width, uint32_t height, const float eye[3],
                                     const float target[3], float fovDeg)
{
    if (!p || !eye || !target || width == 0 || height == 0 || !(fovDeg > 0.0f && fovDeg < 180.0f))
        return sb::fail(STRELKA_ERR_INVALID_ARGUMENT, "invalid camera arguments");
    const double e[3] = {eye[0], eye[1], eye[2]}, t[3] = {target[0], target[1], target[2]};
    if (e[0] == t[0] && e[1] == t[1] && e[2] == t[2]) return sb::fail(STRELKA_ERR_INVALID_ARGUMENT, "eye == target");
    PathTracerParam c;
    set_camera(c, width, height, e, t, fovDeg);
    p->viewToWorld = c.viewToWorld;
    p->clipToView = c.clipToView;
    p->viewToClip = c.viewToClip;
    p->worldToView = c.worldToView;
    p->camPos = c.camPos;
    p->dimension[0] = c.dimension[0];
    p->dimension[1] = c.dimension[1];
    p->invDimension[0] = c.invDimension[0];
    p->invDimension[1] = c.invDimension[1];
    return STRELKA_OK;
}

extern "C" void strelka_scene_free(StrelkaHostScene* s)
{
    if (!s) return;
    free(s->vb);
    free(s->ib);
    free(s->instances);
    free(s->lights);
    free(s->materials);
    free(s->argBlock);
    free(s->resourceInfos);
    if (s->textures)
        for (uint32_t i = 0; i < s->numTextures; ++i) free(s->textures[i]);
    free(s->textures);
    free(s->texWidth);
    free(s->texHeight);
    free(s->envRGBA);
    free(s->envMarginalCdf);
    free(s->envConditionalCdf);
    free(s->nodes);
    memset(s, 0, sizeof(*s));
}
