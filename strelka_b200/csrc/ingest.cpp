// ingest.cpp — the data formats on the host side of the path: vertex packing
// of the Hydra render delegate (src/hdStrelka/RenderPass.cpp:50-126) and the
// translation of USD light parameters into the shader's UniformLight
// (src/hdStrelka/Light.cpp:112-198 with src/scene/scene.cpp:459-511), so
// scenes exported from a USD stage can be replayed through this library.
//
// Arithmetic is float32 in the reference's order.  glm evaluates a matrix x
// vector product column-pairwise, ((c0 x + c1 y) + (c2 z + c3 w)); the
// products below follow that order.
#include <cmath>
#include <cstring>

#include "common.h"

namespace {

// column-major 4x4 (m[4*c + r]) times (x, y, z, w), pairwise like glm
void mat_vec(const float* m, const float v[4], float out[4])
{
    for (int r = 0; r < 4; ++r) {
        const float a = m[0 + r] * v[0] + m[4 + r] * v[1];
        const float b = m[8 + r] * v[2] + m[12 + r] * v[3];
        out[r] = a + b;
    }
}

// a * b (both column-major): column c of the product is a * (column c of b)
void mat_mul(const float* a, const float* b, float* out)
{
    float t[16];
    for (int c = 0; c < 4; ++c) mat_vec(a, b + 4 * c, t + 4 * c);
    memcpy(out, t, sizeof(t));
}

void scale_matrix(float sx, float sy, float sz, float* m)
{
    memset(m, 0, 16 * sizeof(float));
    m[0] = sx;
    m[5] = sy;
    m[10] = sz;
    m[15] = 1.0f;
}

void store(StrelkaFloat4& d, const float v[4])
{
    d.x = v[0];
    d.y = v[1];
    d.z = v[2];
    d.w = v[3];
}

// Colour of a black body, 1000 K .. 10000 K in 500 K steps, Rec. 709
// primaries: the table of John Walker's "Colour Rendering of Spectra"
// (specrend.c) that the reference interpolates, with the first and last
// knots repeated (Light.cpp:15-57).
const float kBlackbody[22][3] = {
    {1.000000f, 0.027490f, 0.000000f}, {1.000000f, 0.027490f, 0.000000f}, {1.000000f, 0.149664f, 0.000000f},
    {1.000000f, 0.256644f, 0.008095f}, {1.000000f, 0.372033f, 0.067450f}, {1.000000f, 0.476725f, 0.153601f},
    {1.000000f, 0.570376f, 0.259196f}, {1.000000f, 0.653480f, 0.377155f}, {1.000000f, 0.726878f, 0.501606f},
    {1.000000f, 0.791543f, 0.628050f}, {1.000000f, 0.848462f, 0.753228f}, {1.000000f, 0.898581f, 0.874905f},
    {1.000000f, 0.942771f, 0.991642f}, {0.906947f, 0.890456f, 1.000000f}, {0.828247f, 0.841838f, 1.000000f},
    {0.765791f, 0.801896f, 1.000000f}, {0.715255f, 0.768579f, 1.000000f}, {0.673683f, 0.740423f, 1.000000f},
    {0.638992f, 0.716359f, 1.000000f}, {0.609681f, 0.695588f, 1.000000f}, {0.609681f, 0.695588f, 1.000000f},
    {0.609681f, 0.695588f, 1.000000f}};

}  // namespace

// RenderPass.cpp:50-56: each component mapped from [-1, 1] to 9 bits
extern "C" uint32_t strelka_pack_normal(const float n[3])
{
    uint32_t packed = (uint32_t)((n[0] + 1.0f) / 2.0f * 511.99999f);
    packed += (uint32_t)((n[1] + 1.0f) / 2.0f * 511.99999f) << 10;
    packed += (uint32_t)((n[2] + 1.0f) / 2.0f * 511.99999f) << 20;
    return packed;
}

// RenderPass.cpp:58-64: each component mapped from [-10, 10] to 14 bits
extern "C" uint32_t strelka_pack_uv(const float uv[2])
{
    int32_t packed = (int32_t)(uint32_t)((uv[0] + 10.0f) / 20.0f * 16383.99999f);
    packed += (int32_t)((uint32_t)((uv[1] + 10.0f) / 20.0f * 16383.99999f) << 16);
    return (uint32_t)packed;
}

// HdStrelkaRenderPass::_BakeMeshInstance (RenderPass.cpp:66-126): positions
// as given, normals packed, texture coordinates with v flipped (1 - v) then
// packed, tangents 0; the mass centre is the float32 running sum / count.
extern "C" int strelka_bake_vertices(const float* points, const float* normals, const float* uvs, uint32_t count,
                                     Vertex* out, float massCenter[3])
{
    if (count && (!points || !normals || !out)) return sb::fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    float sum[3] = {0.0f, 0.0f, 0.0f};
    for (uint32_t j = 0; j < count; ++j) {
        Vertex& v = out[j];
        memset(&v, 0, sizeof(v));
        for (int a = 0; a < 3; ++a) {
            v.position[a] = points[3 * (size_t)j + a];
            sum[a] += v.position[a];
        }
        v.normal = strelka_pack_normal(normals + 3 * (size_t)j);
        if (uvs) {
            const float uv[2] = {uvs[2 * (size_t)j], 1.0f - uvs[2 * (size_t)j + 1]};
            v.uv = strelka_pack_uv(uv);
        }
    }
    if (massCenter) {
        for (int a = 0; a < 3; ++a) massCenter[a] = count ? sum[a] / (float)count : 0.0f;
    }
    return STRELKA_OK;
}

// _BlackbodyTemperatureAsRgb (Light.cpp:59-98): uniform Catmull-Rom spline
// through the table, normalised to the Rec. 709 luma of (1, 1, 1), negative
// components clamped to 0.
extern "C" int strelka_blackbody_rgb(float kelvin, float rgb[3])
{
    if (!rgb) return sb::fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    float u = (kelvin - 1000.0f) / 9000.0f;
    u = u < 0.0f ? 0.0f : (u > 1.0f ? 1.0f : u);
    const int numSegs = 22 - 4;
    const float x = u * (float)numSegs;
    const int seg = (int)std::floor(x);
    const float t = x - (float)seg;
    // Catmull-Rom basis rows: a, b, c, d of a t^3 + b t^2 + c t + d
    static const float B[4][4] = {
        {-0.5f, 1.5f, -1.5f, 0.5f}, {1.0f, -2.5f, 2.0f, -0.5f}, {-0.5f, 0.0f, 0.5f, 0.0f}, {0.0f, 1.0f, 0.0f, 0.0f}};
    float out[3];
    for (int ch = 0; ch < 3; ++ch) {
        float coef[4];
        for (int r = 0; r < 4; ++r)
            coef[r] = ((B[r][0] * kBlackbody[seg][ch] + B[r][1] * kBlackbody[seg + 1][ch]) + B[r][2] * kBlackbody[seg + 2][ch]) +
                      B[r][3] * kBlackbody[seg + 3][ch];
        out[ch] = ((coef[0] * t + coef[1]) * t + coef[2]) * t + coef[3];
    }
    const float luma = (out[0] * 0.2126f + out[1] * 0.7152f) + out[2] * 0.0722f;
    for (int ch = 0; ch < 3; ++ch) {
        const float v = out[ch] / luma;
        rgb[ch] = v > 0.0f ? v : 0.0f;
    }
    return STRELKA_OK;
}

// HdStrelkaLight::Sync (Light.cpp:112-198) then Scene::updateLight
// (scene.cpp:459-511): colour x black body (when enabled), intensity x
// 2^clamp(exposure, -50, 50), the shape packed into UniformLight, and the
// colour scaled by intensity / area (colour.w = that factor).
extern "C" int strelka_light_from_usd(const StrelkaUsdLight* in, UniformLight* out)
{
    if (!in || !out) return sb::fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    if (in->type > 2) return sb::fail(STRELKA_ERR_INVALID_ARGUMENT, "unknown light type %u", in->type);
    float color[3] = {in->color[0], in->color[1], in->color[2]};
    if (in->enableColorTemperature) {
        float bb[3];
        strelka_blackbody_rgb(in->colorTemperature, bb);
        for (int a = 0; a < 3; ++a) color[a] *= bb[a];
    }
    float exposure = in->exposure;
    exposure = exposure < -50.0f ? -50.0f : (exposure > 50.0f ? 50.0f : exposure);
    const float intensity = in->intensity * powf(2.0f, exposure);
    memset(out, 0, sizeof(*out));
    const float* xf = in->xform;
    float local[16], s[16];
    float perArea = intensity;
    if (in->type == 0) {
        scale_matrix(in->width, in->height, 1.0f, s);
        mat_mul(xf, s, local);
        const float c[4][4] = {{0.5f, 0.5f, 0.0f, 1.0f}, {-0.5f, 0.5f, 0.0f, 1.0f}, {-0.5f, -0.5f, 0.0f, 1.0f},
                               {0.5f, -0.5f, 0.0f, 1.0f}};
        for (int k = 0; k < 4; ++k) {
            float p[4];
            mat_vec(local, c[k], p);
            store(out->points[k], p);
        }
        perArea /= (in->width * in->height);
    } else {
        const float radius = in->radius * xf[0];  // Light.cpp:190, uniform scale
        if (in->type == 1) {
            scale_matrix(radius, radius, radius, s);
            mat_mul(xf, s, local);
            const float r4[4] = {radius, 0.0f, 0.0f, 0.0f};
            const float o[4] = {0.0f, 0.0f, 0.0f, 1.0f}, ax[4] = {1.0f, 0.0f, 0.0f, 0.0f},
                        ay[4] = {0.0f, 1.0f, 0.0f, 0.0f}, az[4] = {0.0f, 0.0f, 1.0f, 0.0f};
            float p[4];
            store(out->points[0], r4);
            mat_vec(local, o, p);
            store(out->points[1], p);
            mat_vec(local, ax, p);
            store(out->points[2], p);
            mat_vec(local, ay, p);
            store(out->points[3], p);
            mat_vec(local, az, p);
            store(out->normal, p);
            perArea /= ((float)M_PI * radius * radius);
        } else {
            scale_matrix(1.0f, 1.0f, 1.0f, s);
            mat_mul(s, xf, local);
            const float r4[4] = {radius, 0.0f, 0.0f, 0.0f};
            const float o[4] = {0.0f, 0.0f, 0.0f, 1.0f};
            float p[4];
            store(out->points[0], r4);
            mat_vec(local, o, p);
            store(out->points[1], p);
            perArea /= (4.0f * (float)M_PI * radius * radius);
        }
    }
    out->type = (int32_t)in->type;
    const float c4[4] = {color[0] * perArea, color[1] * perArea, color[2] * perArea, 1.0f * perArea};
    store(out->color, c4);
    return STRELKA_OK;
}
