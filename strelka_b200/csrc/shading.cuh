// shading.cuh — camera rays, light sampling, native BSDFs and the per-bounce
// shading step of shaders/pathtracerMdl.hlsl, sm_100a.
//
// The bounce is split into shade() and apply_shadow() so the megakernel and
// the wavefront kernels run the same code: shade() performs everything of
// one loop iteration of pathTraceCameraRays (pathtracerMdl.hlsl:222-401)
// except the shadow-ray query, and returns the next-event contribution the
// reference would add when the light is visible.  With visibility 0 the
// reference adds exactly +/-0 whenever that contribution's inputs are finite,
// so the shadow query can be deferred; when they are not finite shade()
// traces the shadow ray itself, keeping every NaN/Inf case identical.
#pragma once
#include "traverse.cuh"

namespace sb {

// ---------------------------------------------------------------------------
// lights.h
struct LightSample {
    v3 pointOnLight;
    float pdf;
    v3 normal;
    float area;
    v3 L;
    float distToLight;
};

__device__ __forceinline__ v3 lp(const UniformLight& l, int i) { return V(l.points[i].x, l.points[i].y, l.points[i].z); }

// lights.h:34-46
__device__ __forceinline__ void frisvad(v3 n, v3& b1, v3& b2)
{
    if (n.z < -0.9999999f) {
        b1 = V(0.0f, -1.0f, 0.0f);
        b2 = V(-1.0f, 0.0f, 0.0f);
        return;
    }
    const float a = 1.0f / (1.0f + n.z);
    const float b = -n.x * n.y * a;
    b1 = V(1.0f - n.x * n.x * a, b, -n.x);
    b2 = V(b, 1.0f - n.y * n.y * a, -n.y);
}

// lights.h:59-89 (the shadowed 'u' and the missing centre are kept)
__device__ __forceinline__ v3 sample_sphere_solid_angle(const UniformLight& l, v3 hitPoint)
{
    v3 c = lp(l, 1);
    float r = l.points[0].x;
    v3 w = vsub(c, hitPoint);
    float distanceToCenter = vlength(w);
    w = vscale(w, 1.0f / distanceToCenter);
    float q = sqrtf(1.0f - (r / distanceToCenter) * (r / distanceToCenter));
    v3 v, u;
    frisvad(w, v, u);
    float r0 = u.x;
    float r1 = u.y;
    float theta = own_acosf(1.0f - r0 + r0 * q);
    float phi = SB_TWO_PI_F * r1;
    float st, ct, sp, cp;
    own_sincos(theta, &st, &ct);
    own_sincos(phi, &sp, &cp);
    v3 local;
    local.x = 5.0f * sp * st;
    local.z = -5.0f * sp * ct;
    local.y = 5.0f * cp;
    return V((local.x * u.x + local.y * w.x) + local.z * v.x, (local.x * u.y + local.y * w.y) + local.z * v.y,
             (local.x * u.z + local.y * w.z) + local.z * v.z);
}

struct SphQuad {
    v3 o, x, y, z;
    float z0, z0sq, x0, y0, y0sq, x1, y1, y1sq, b0, b1, b0sq, k, S;
};

// lights.h:102-166
__device__ __forceinline__ SphQuad sphquad_init(const UniformLight& l, v3 o)
{
    SphQuad q;
    v3 p0 = lp(l, 0), p1 = lp(l, 1), p3 = lp(l, 3);
    v3 ex = vsub(p1, p0);
    v3 ey = vsub(p3, p0);
    v3 s = p0;
    float exl = vlength(ex);
    float eyl = vlength(ey);
    q.o = o;
    q.x = vdivs(ex, exl);
    q.y = vdivs(ey, eyl);
    q.z = vcross(q.x, q.y);
    v3 d = vsub(s, o);
    q.z0 = vdot(d, q.z);
    if (q.z0 > 0) {
        q.z = vscale(q.z, -1.0f);
        q.z0 *= -1.0f;
    }
    q.z0sq = q.z0 * q.z0;
    q.x0 = vdot(d, q.x);
    q.y0 = vdot(d, q.y);
    q.x1 = q.x0 + exl;
    q.y1 = q.y0 + eyl;
    q.y0sq = q.y0 * q.y0;
    q.y1sq = q.y1 * q.y1;
    v3 v00 = V(q.x0, q.y0, q.z0), v01 = V(q.x0, q.y1, q.z0), v10 = V(q.x1, q.y0, q.z0), v11 = V(q.x1, q.y1, q.z0);
    v3 n0 = vnormalize(vcross(v00, v10));
    v3 n1 = vnormalize(vcross(v10, v11));
    v3 n2 = vnormalize(vcross(v11, v01));
    v3 n3 = vnormalize(vcross(v01, v00));
    float g0 = own_acosf(-vdot(n0, n1));
    float g1 = own_acosf(-vdot(n1, n2));
    float g2 = own_acosf(-vdot(n2, n3));
    float g3 = own_acosf(-vdot(n3, n0));
    q.b0 = n0.z;
    q.b1 = n2.z;
    q.b0sq = q.b0 * q.b0;
    q.k = SB_TWO_PI_F - g2 - g3;
    q.S = g0 + g1 - q.k;
    return q;
}

// lights.h:168-194
__device__ __forceinline__ v3 sphquad_sample(const SphQuad& q, float u, float v)
{
    float au = u * q.S + q.k;
    float sau, cau;
    own_sincos(au, &sau, &cau);
    float fu = (cau * q.b0 - q.b1) / sau;
    float cu = 1.0f / sqrtf(fu * fu + q.b0sq) * (fu > 0 ? 1.0f : -1.0f);
    cu = fminf(fmaxf(cu, -1.0f), 1.0f);
    float xu = -(cu * q.z0) / sqrtf(1.0f - cu * cu);
    xu = fminf(fmaxf(xu, q.x0), q.x1);
    float d = sqrtf(xu * xu + q.z0sq);
    float h0 = q.y0 / sqrtf(d * d + q.y0sq);
    float h1 = q.y1 / sqrtf(d * d + q.y1sq);
    float hv = h0 + v * (h1 - h0);
    float hv2 = hv * hv;
    float eps = 1e-5f;
    float yv = (hv < 1.0f - eps) ? (hv * d) / sqrtf(1.0f - hv2) : q.y1;
    return vadd(vadd(vadd(q.o, vscale(q.x, xu)), vscale(q.y, yv)), vscale(q.z, q.z0));
}

// lights.h:196-219
__device__ __forceinline__ void concentric_sample_disk(float ux, float uy, float& ox, float& oy)
{
    float x = 2.0f * ux - 1.0f;
    float y = 2.0f * uy - 1.0f;
    if (x == 0 && y == 0) { ox = 0.0f; oy = 0.0f; return; }
    float theta, r;
    if (fabsf(x) > fabsf(y)) {
        r = x;
        theta = SB_PI_OVER_4_F * (y / x);
    } else {
        r = y;
        theta = SB_PI_OVER_2_F - SB_PI_OVER_4_F * (x / y);
    }
    float s, c;
    own_sincos(theta, &s, &c);
    ox = r * c;
    oy = r * s;
}

// lights.h:230-282
__device__ __forceinline__ v3 light_normal(const UniformLight& l, v3 hitPoint)
{
    v3 norm = V(0.0f, 0.0f, 0.0f);
    if (l.type == 0) {
        v3 e1 = vsub(lp(l, 1), lp(l, 0));
        v3 e2 = vsub(lp(l, 3), lp(l, 0));
        norm = vneg(vnormalize(vcross(e1, e2)));
    } else if (l.type == 1) {
        norm = V(l.normal.x, l.normal.y, l.normal.z);
    } else if (l.type == 2) {
        norm = vnormalize(vsub(hitPoint, lp(l, 1)));
    }
    return norm;
}
__device__ __forceinline__ float light_area(const UniformLight& l)
{
    float area = 0.0f;
    if (l.type == 0) {
        v3 e1 = vsub(lp(l, 1), lp(l, 0));
        v3 e2 = vsub(lp(l, 3), lp(l, 0));
        area = vlength(vcross(e1, e2));
    } else if (l.type == 1) {
        area = SB_PI_F * l.points[0].x * l.points[0].x;
    } else if (l.type == 2) {
        area = SB_FOUR_PI_F * l.points[0].x * l.points[0].x;
    }
    return area;
}
__device__ __forceinline__ void fill_light_data(const UniformLight& l, v3 hitPoint, LightSample& ls)
{
    ls.area = light_area(l);
    ls.normal = light_normal(l, hitPoint);
    v3 toLight = vsub(ls.pointOnLight, hitPoint);
    float len = vlength(toLight);
    ls.L = vdivs(toLight, len);
    ls.distToLight = len;
}

// lights.h:284-340
__device__ __forceinline__ LightSample sample_light(const UniformLight& l, v3 hitPoint, float ux, float uy)
{
    LightSample ls;
    ls.pointOnLight = V(0.0f, 0.0f, 0.0f);
    ls.pdf = 0.0f;
    ls.normal = V(0.0f, 0.0f, 0.0f);
    ls.area = 0.0f;
    ls.L = V(0.0f, 0.0f, 0.0f);
    ls.distToLight = 0.0f;
    if (l.type == 0) {
        SphQuad q = sphquad_init(l, hitPoint);
        ls.pointOnLight = sphquad_sample(q, ux, uy);
        fill_light_data(l, hitPoint, ls);
        ls.pdf = ls.distToLight * ls.distToLight / (-vdot(ls.L, ls.normal) * ls.area);
    } else if (l.type == 1) {
        float pdx, pdy;
        concentric_sample_disk(ux, uy, pdx, pdy);
        float x = l.points[0].x * pdx;
        float y = l.points[0].x * pdy;
        ls.pointOnLight = vadd(vadd(lp(l, 1), vscale(lp(l, 2), x)), vscale(lp(l, 3), y));
        fill_light_data(l, hitPoint, ls);
        ls.pdf = ls.distToLight * ls.distToLight / (-vdot(ls.L, ls.normal) * ls.area);
    } else if (l.type == 2) {
        ls.pointOnLight = sample_sphere_solid_angle(l, hitPoint);
        fill_light_data(l, hitPoint, ls);
        float distanceToCenter = vlength(vsub(lp(l, 1), hitPoint));
        float sinThetaMax2 = l.points[0].x * l.points[0].x / (distanceToCenter * distanceToCenter);
        float cosThetaMax = sqrtf(fmaxf(0.0f, 1.0f - sinThetaMax2));
        ls.pdf = 1.0f / (SB_TWO_PI_F * (1.0f - cosThetaMax));
    }
    return ls;
}

// ---------------------------------------------------------------------------
// Environment light (extension; the reference's miss adds zero).
__device__ __forceinline__ float own_atan2(float y, float x)
{
    float r = sqrtf(x * x + y * y);
    if (r == 0.0f) return 0.0f;
    float a = own_acosf(fminf(fmaxf(x / r, -1.0f), 1.0f));
    return y < 0.0f ? -a : a;
}
__device__ __forceinline__ v3 env_lookup(const StrelkaEnvMap& e, v3 d, int& texel)
{
    float phi = own_atan2(d.x, -d.z);
    float u = phi * (1.0f / SB_TWO_PI_F) + 0.5f;
    float v = own_acosf(fminf(fmaxf(d.y, -1.0f), 1.0f)) * SB_INV_PI_F;
    int x = (int)(u * (float)e.width);
    int y = (int)(v * (float)e.height);
    x = x < 0 ? 0 : (x >= (int)e.width ? (int)e.width - 1 : x);
    y = y < 0 ? 0 : (y >= (int)e.height ? (int)e.height - 1 : y);
    texel = y * (int)e.width + x;
    float4 p = __ldg(reinterpret_cast<const float4*>(e.rgba32f) + texel);
    return V(p.x, p.y, p.z);
}
__device__ __forceinline__ float env_pdf(const StrelkaEnvMap& e, int texel, v3 d)
{
    int y = texel / (int)e.width;
    int x = texel - y * (int)e.width;
    const float* cc = e.conditional_cdf + (size_t)y * (e.width + 1);
    float pRow = __ldg(&e.marginal_cdf[y + 1]) - __ldg(&e.marginal_cdf[y]);
    float pCol = __ldg(&cc[x + 1]) - __ldg(&cc[x]);
    float sinTheta = sqrtf(fmaxf(0.0f, 1.0f - d.y * d.y));
    if (!(sinTheta > 0.0f)) return 0.0f;
    float texelSolidAngle = (SB_TWO_PI_F / (float)e.width) * (SB_PI_F / (float)e.height) * sinTheta;
    return pRow * pCol / texelSolidAngle;
}
// The index lo in [0, n) with cdf[lo] <= u < cdf[lo + 1] (lo = 0 below
// cdf[1], n - 1 at or above cdf[n - 1]).  Both forms keep the invariant
// "lo == 0 or cdf[lo] <= u, and hi == n or cdf[hi] > u" and stop at
// hi == lo + 1, which for a non-decreasing CDF leaves one possible lo, so the
// four-way form returns the binary search's index.  It compares u with three
// cut points per level, loaded together: about half as many dependent loads
// (11 instead of 19 for a 512-row marginal and a 1024-column row).
__device__ __forceinline__ int upper_bound_cdf(const float* cdf, int n, float u)
{
    int lo = 0, hi = n;
    while (hi - lo > 4) {
        const int step = (hi - lo) >> 2;
        const int m1 = lo + step, m2 = m1 + step, m3 = m2 + step;
        const float c1 = __ldg(&cdf[m1]), c2 = __ldg(&cdf[m2]), c3 = __ldg(&cdf[m3]);
        if (c3 <= u) {
            lo = m3;
        } else if (c2 <= u) {
            lo = m2;
            hi = m3;
        } else if (c1 <= u) {
            lo = m1;
            hi = m2;
        } else {
            hi = m1;
        }
    }
    while (lo + 1 < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(&cdf[mid]) <= u) lo = mid; else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ v3 env_sample(const StrelkaEnvMap& e, float u1, float u2, float& pdf, v3& radiance)
{
    int y = upper_bound_cdf(e.marginal_cdf, (int)e.height, u1);
    const float* cc = e.conditional_cdf + (size_t)y * (e.width + 1);
    int x = upper_bound_cdf(cc, (int)e.width, u2);
    float m0 = __ldg(&e.marginal_cdf[y]), m1 = __ldg(&e.marginal_cdf[y + 1]);
    float c0 = __ldg(&cc[x]), c1 = __ldg(&cc[x + 1]);
    float fy = (u1 - m0) / fmaxf(m1 - m0, 1e-30f);
    float fx = (u2 - c0) / fmaxf(c1 - c0, 1e-30f);
    float v = ((float)y + fsat(fy)) / (float)e.height;
    float u = ((float)x + fsat(fx)) / (float)e.width;
    float theta = v * SB_PI_F;
    float phi = (u - 0.5f) * SB_TWO_PI_F;
    float st, ct, sp, cp;
    own_sincos(theta, &st, &ct);
    own_sincos(phi, &sp, &cp);
    v3 d = V(st * sp, ct, -(st * cp));
    int texel = y * (int)e.width + x;
    float4 p = __ldg(reinterpret_cast<const float4*>(e.rgba32f) + texel);
    radiance = V(p.x, p.y, p.z);
    pdf = env_pdf(e, texel, d);
    return d;
}

// ---------------------------------------------------------------------------
// Native materials (StrelkaMaterialArgs records in the MDL argument block).
struct ShadeState {
    v3 normal, geom_normal, position;
    float u, v;
};
struct Mat {
    v3 base;
    float roughness;
    v3 emission;
    float ior;
    uint32_t tex;
    int fn;
};

__device__ __forceinline__ int wrapi(int i, int n) { int r = i % n; return r < 0 ? r + n : r; }

// mdl_runtime.hlsl:125-140 (smootherstep) + bilinear REPEAT over sRGB texels
__device__ __forceinline__ void tex_lookup(const DevScene& s, const StrelkaTexture& t, float u, float v, float out[4])
{
    float W = (float)t.width, H = (float)t.height;
    float rx = u * W + 0.5f, ry = v * H + 0.5f;
    float ui = floorf(rx), vi = floorf(ry);
    float uf = rx - ui, vf = ry - vi;
    uf = uf * uf * uf * (uf * (uf * 6.0f - 15.0f) + 10.0f);
    vf = vf * vf * vf * (vf * (vf * 6.0f - 15.0f) + 10.0f);
    rx = ui + uf;
    ry = vi + vf;
    float cu = (rx - 0.5f) / W, cv = (ry - 0.5f) / H;
    float x = cu * W - 0.5f, y = cv * H - 0.5f;
    float x0f = floorf(x), y0f = floorf(y);
    float fx = x - x0f, fy = y - y0f;
    int x0 = wrapi((int)x0f, (int)t.width), y0 = wrapi((int)y0f, (int)t.height);
    int x1 = wrapi(x0 + 1, (int)t.width), y1 = wrapi(y0 + 1, (int)t.height);
    const uchar4* px = reinterpret_cast<const uchar4*>(t.rgba8);
    uchar4 p00 = __ldg(&px[(size_t)y0 * t.width + x0]);
    uchar4 p10 = __ldg(&px[(size_t)y0 * t.width + x1]);
    uchar4 p01 = __ldg(&px[(size_t)y1 * t.width + x0]);
    uchar4 p11 = __ldg(&px[(size_t)y1 * t.width + x1]);
    const unsigned char c00[4] = {p00.x, p00.y, p00.z, p00.w};
    const unsigned char c10[4] = {p10.x, p10.y, p10.z, p10.w};
    const unsigned char c01[4] = {p01.x, p01.y, p01.z, p01.w};
    const unsigned char c11[4] = {p11.x, p11.y, p11.z, p11.w};
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float a00 = c < 3 ? __ldg(&s.srgbLut[c00[c]]) : (float)c00[c] / 255.0f;
        float a10 = c < 3 ? __ldg(&s.srgbLut[c10[c]]) : (float)c10[c] / 255.0f;
        float a01 = c < 3 ? __ldg(&s.srgbLut[c01[c]]) : (float)c01[c] / 255.0f;
        float a11 = c < 3 ? __ldg(&s.srgbLut[c11[c]]) : (float)c11[c] / 255.0f;
        float top = a00 + fx * (a10 - a00);
        float bot = a01 + fx * (a11 - a01);
        out[c] = top + fy * (bot - top);
    }
}

__device__ __forceinline__ bool load_material(const DevScene& s, int32_t materialId, const ShadeState& st, Mat& m)
{
    if (materialId < 0 || (uint32_t)materialId >= s.numMaterials) return false;
    const MdlMaterial mm = s.materials[materialId];
    if (mm.arg_block_offset < 0 || (uint64_t)mm.arg_block_offset + sizeof(StrelkaMaterialArgs) > s.argBlockBytes ||
        (mm.arg_block_offset & 15) != 0)
        return false;
    if (mm.functionId < 0 || mm.functionId >= STRELKA_FN_COUNT) return false;
    const float4* a = reinterpret_cast<const float4*>(s.argBlock + mm.arg_block_offset);
    float4 a0 = __ldg(a), a1 = __ldg(a + 1);
    uint4 a2 = __ldg(reinterpret_cast<const uint4*>(a + 2));
    m.base = V(a0.x, a0.y, a0.z);
    m.roughness = a0.w;
    m.emission = V(a1.x, a1.y, a1.z);
    m.ior = a1.w;
    m.tex = a2.x;
    m.fn = mm.functionId;
    if (m.tex != 0) {
        if (m.tex - 1 >= s.numResInfos) return false;
        uint32_t slot = s.resInfos[m.tex - 1].gpu_resource_array_start;
        if (slot >= s.numTextures) return false;
        float texel[4];
        tex_lookup(s, s.textures[slot], st.u, st.v, texel);
        m.base = V(m.base.x * texel[0], m.base.y * texel[1], m.base.z * texel[2]);
    }
    return true;
}

__device__ __forceinline__ float ggx_d(float alpha, float noh)
{
    float a2 = alpha * alpha;
    float t = noh * noh * (a2 - 1.0f) + 1.0f;
    return a2 / (SB_PI_F * t * t);
}
__device__ __forceinline__ float ggx_g1(float alpha, float nov)
{
    float a2 = alpha * alpha;
    return 2.0f * nov / (nov + sqrtf(a2 + (1.0f - a2) * nov * nov));
}
__device__ __forceinline__ float mat_alpha(float roughness) { return fmaxf(roughness * roughness, 1e-3f); }
__device__ __forceinline__ float schlick_weight(float c)
{
    float m = fsat(1.0f - c);
    float m2 = m * m;
    return m2 * m2 * m;
}
__device__ __forceinline__ float fresnel_dielectric(float cosi, float eta)
{
    float sin2t = eta * eta * (1.0f - cosi * cosi);
    if (sin2t >= 1.0f) return 1.0f;
    float cost = sqrtf(fsat(1.0f - sin2t));
    float rs = (cosi - eta * cost) / (cosi + eta * cost);
    float rp = (eta * cosi - cost) / (eta * cosi + cost);
    return 0.5f * (rs * rs + rp * rp);
}
__device__ __forceinline__ v3 schlick_f(v3 f0, float w)
{
    return V(f0.x + (1.0f - f0.x) * w, f0.y + (1.0f - f0.y) * w, f0.z + (1.0f - f0.z) * w);
}

struct EvalOut {
    v3 bsdf_diffuse, bsdf_glossy;
    float pdf;
};
struct SampleOut {
    v3 k2, bsdf_over_pdf;
    float pdf;
    int event;
};

// mdl_bsdf_scattering_evaluate contract (values include the cosine);
// Lambert as shaders/pathtracer.hlsl:176-185.
__device__ __forceinline__ EvalOut bsdf_evaluate(const Mat& m, const ShadeState& st, v3 k1, v3 k2, float ior1, float ior2)
{
    EvalOut e;
    e.bsdf_diffuse = V(0.0f, 0.0f, 0.0f);
    e.bsdf_glossy = V(0.0f, 0.0f, 0.0f);
    e.pdf = 0.0f;
    v3 N = st.normal;
    if (m.fn == STRELKA_FN_LAMBERT) {
        float c = fsat(vdot(N, k2));
        e.bsdf_diffuse = vscale(m.base, SB_INV_PI_F * c);
        e.pdf = SB_INV_PI_F * (c + 1e-6f);
        return e;
    }
    float nol = vdot(N, k2), nov = vdot(N, k1);
    if (!(nol > 0.0f) || !(nov > 0.0f)) return e;
    v3 h = vnormalize(vadd(k1, k2));
    float noh = fsat(vdot(N, h)), voh = fsat(vdot(k1, h));
    float alpha = mat_alpha(m.roughness);
    float D = ggx_d(alpha, noh);
    float G = ggx_g1(alpha, nov) * ggx_g1(alpha, nol);
    if (m.fn == STRELKA_FN_GGX_CONDUCTOR) {
        v3 F = schlick_f(m.base, schlick_weight(voh));
        float k = D * G / (4.0f * nov);
        e.bsdf_glossy = vscale(F, k);
        e.pdf = D * noh / (4.0f * voh);
    } else {
        float i1 = ior1 < 0.0f ? m.ior : ior1;
        float i2 = ior2 < 0.0f ? m.ior : ior2;
        float F = fresnel_dielectric(voh, i1 / i2);
        float k = F * D * G / (4.0f * nov);
        e.bsdf_glossy = V(k, k, k);
        e.pdf = F * D * noh / (4.0f * voh);
    }
    return e;
}

// mdl_bsdf_scattering_sample contract; Lambert as
// shaders/pathtracer.hlsl:208-234 with helper.h:41-50,73-79.
__device__ __forceinline__ SampleOut bsdf_sample(const Mat& m, const ShadeState& st, v3 k1, const float xi[4], float ior1,
                                                 float ior2)
{
    SampleOut so;
    so.k2 = V(0.0f, 0.0f, 0.0f);
    so.bsdf_over_pdf = V(0.0f, 0.0f, 0.0f);
    so.pdf = 0.0f;
    so.event = SB_EV_ABSORB;
    v3 N = st.normal;
    Frame f = tangent_space(N);
    if (m.fn == STRELKA_FN_LAMBERT) {
        v3 w = sample_hemisphere_cosine(xi[0], xi[1]);
        so.k2 = frame_to_world(f, w);
        so.pdf = SB_INV_PI_F * (fsat(vdot(N, so.k2)) + 1e-6f);
        so.bsdf_over_pdf = m.base;
        so.event = SB_EV_DIFFUSE | SB_EV_REFLECTION;
        return so;
    }
    float nov = vdot(N, k1);
    if (!(nov > 0.0f)) return so;
    float alpha = mat_alpha(m.roughness);
    float a2 = alpha * alpha;
    float cosThetaH = sqrtf((1.0f - xi[0]) / (xi[0] * (a2 - 1.0f) + 1.0f));
    float sinThetaH = sqrtf(fsat(1.0f - cosThetaH * cosThetaH));
    float phi = SB_TWO_PI_F * xi[1];
    float sp, cp;
    own_sincos(phi, &sp, &cp);
    v3 h = frame_to_world(f, V(cp * sinThetaH, sp * sinThetaH, cosThetaH));
    float voh = vdot(k1, h);
    if (!(voh > 0.0f)) return so;
    float noh = fsat(vdot(N, h));
    float G1v = ggx_g1(alpha, nov);
    if (m.fn == STRELKA_FN_GGX_CONDUCTOR) {
        so.k2 = vsub(vscale(h, 2.0f * voh), k1);
        float nol = vdot(N, so.k2);
        if (!(nol > 0.0f)) return so;
        v3 F = schlick_f(m.base, schlick_weight(voh));
        float G = G1v * ggx_g1(alpha, nol);
        float k = G * voh / (nov * noh);
        so.bsdf_over_pdf = vscale(F, k);
        so.pdf = ggx_d(alpha, noh) * noh / (4.0f * voh);
        so.event = SB_EV_GLOSSY | SB_EV_REFLECTION;
        return so;
    }
    float i1 = ior1 < 0.0f ? m.ior : ior1;
    float i2 = ior2 < 0.0f ? m.ior : ior2;
    float eta = i1 / i2;
    float F = fresnel_dielectric(voh, eta);
    float D = ggx_d(alpha, noh);
    if (xi[2] < F) {
        so.k2 = vsub(vscale(h, 2.0f * voh), k1);
        float nol = vdot(N, so.k2);
        if (!(nol > 0.0f)) return so;
        float G = G1v * ggx_g1(alpha, nol);
        float k = G * voh / (nov * noh);
        so.bsdf_over_pdf = V(k, k, k);
        so.pdf = F * D * noh / (4.0f * voh);
        so.event = SB_EV_GLOSSY | SB_EV_REFLECTION;
        return so;
    }
    float sin2t = eta * eta * (1.0f - voh * voh);
    float c2 = sqrtf(fsat(1.0f - sin2t));
    float sc = eta * voh - c2;
    so.k2 = vadd(vscale(k1, -eta), vscale(h, sc));
    so.k2 = vnormalize(so.k2);
    float nol = vdot(N, so.k2);
    if (!(nol < 0.0f)) { so.event = SB_EV_ABSORB; return so; }
    float G = G1v * ggx_g1(alpha, -nol);
    float k = G * voh / (nov * noh);
    so.bsdf_over_pdf = vscale(m.base, k);
    so.pdf = (1.0f - F) * D * noh;
    so.event = SB_EV_GLOSSY | SB_EV_TRANSMISSION;
    return so;
}

// ---------------------------------------------------------------------------
// Camera, pathtracerMdl.hlsl:94-202
__device__ __forceinline__ void stratified_optimized(uint32_t sIn, float& rx, float& ry)
{
    const int N = 16, p = 16;
    const int m = 4;
    const int n = (N + m - 1) / m;
    int s = (int)permute(sIn, (uint32_t)N, (uint32_t)p * 0x51633e2du);
    int sx = (int)permute((uint32_t)(s % m), (uint32_t)m, (uint32_t)p * 0x68bc21ebu);
    int sy = (int)permute((uint32_t)(s / m), (uint32_t)n, (uint32_t)p * 0x02e5be93u);
    float jx = randfloat((uint32_t)s, (uint32_t)p * 0x967a889bu);
    float jy = randfloat((uint32_t)s, (uint32_t)p * 0x368cc8b7u);
    rx = ((float)sx + ((float)sy + jx) / (float)n) / (float)m;
    ry = ((float)s + jy) / (float)N;
}
__device__ __forceinline__ void stratified1(uint32_t s, uint32_t& rng, float& jx, float& jy)
{
    const int m = 4;
    const int n = (16 + m - 1) / m;
    uint32_t x = (s / (uint32_t)n) % (uint32_t)n;
    uint32_t y = (s % (uint32_t)m) % (uint32_t)m;
    float r0 = rand01(rng);
    jx = ((float)x + ((float)y + r0) / (float)n) / (float)m;
    float r1 = rand01(rng);
    jy = ((float)y + ((float)x + r1) / (float)m) / (float)n;
}
__device__ __forceinline__ void camera_ray(const PathTracerParam& ubo, uint32_t px, uint32_t py, uint32_t& rng, uint32_t s,
                                           v3& o, v3& d)
{
    float ppx = 0.0f, ppy = 0.0f;
    if (ubo.stratifiedSamplingType == 0) {
        ppx = (float)px + 0.5f;
        ppy = (float)py + 0.5f;
    } else if (ubo.stratifiedSamplingType == 1) {
        ppx = (float)px + rand01(rng);
        ppy = (float)py + rand01(rng);
    } else if (ubo.stratifiedSamplingType == 2) {
        float jx, jy;
        stratified1(s, rng, jx, jy);
        ppx = (float)px + jx;
        ppy = (float)py + jy;
    } else if (ubo.stratifiedSamplingType == 3) {
        float jx, jy;
        stratified_optimized(s, jx, jy);
        ppx = (float)px + jx;
        ppy = (float)py + jy;
    }
    float ndcx = (ppx / (float)ubo.dimension[0]) * 2.0f - 1.0f;
    float ndcy = (ppy / (float)ubo.dimension[1]) * 2.0f - 1.0f;
    float clip[4] = {ndcx, ndcy, 1.0f, 1.0f};
    float view[4];
    mat_mul4(ubo.clipToView.m, clip, view);
    float vdir[4] = {view[0], view[1], view[2], 0.0f};
    float wdir[4];
    mat_mul4(ubo.viewToWorld.m, vdir, wdir);
    float orig[4] = {0.0f, 0.0f, 0.0f, 1.0f};
    float wo[4];
    mat_mul4(ubo.viewToWorld.m, orig, wo);
    o = V(wo[0], wo[1], wo[2]);
    d = vnormalize(V(wdir[0], wdir[1], wdir[2]));
}

// ---------------------------------------------------------------------------
// Path state and the bounce.
struct PathState {
    v3 ro;
    float tmax;
    v3 rd;
    float lastPdf;  // pdf of the last BSDF sample (environment MIS only)
    v3 throughput;
    v3 color;
    uint32_t rng;
    int depth;
    int specular;
    int inside;
    int nrcReady;  // radiance cache: the path has made a diffuse-ish bounce
};

// Radiance-cache hook of shade(): mode 1 records the shading vertex (training
// paths), mode 2 also ends the path there with a cache query once the path
// has made a diffuse-ish bounce (a Lambert sample, or roughness >= threshold).
struct NrcShade {
    int mode;
    float diffuseRoughness;
    bool has;
    bool terminate;
    v3 pos, normal;
    float rough;
};

// Deferred next-event contribution (see file comment).
struct ShadowReq {
    int kind;  // 0 none, 1 light (light instances count as visible), 2 environment
    v3 o;
    float tmax;
    v3 d;
    v3 cd, cg;  // contribution to add when visible
};

__device__ __forceinline__ void init_path(const PathTracerParam& ubo, uint64_t idx, PathState& ps)
{
    const uint32_t W = (uint32_t)ubo.dimension[0];
    const uint32_t spp = (uint32_t)ubo.spp;
    const uint32_t px = (uint32_t)idx / spp % W;
    const uint32_t py = (uint32_t)idx / spp / W;
    const uint32_t sampleNum = (uint32_t)idx % spp;
    const uint32_t seedFrame = ubo.frameNumber * spp + sampleNum;
    ps.rng = init_rng(px, py, W, seedFrame);
    camera_ray(ubo, px, py, ps.rng, seedFrame, ps.ro, ps.rd);
    ps.tmax = 1e9f;
    ps.lastPdf = 0.0f;
    ps.throughput = V(1.0f, 1.0f, 1.0f);
    ps.color = V(0.0f, 0.0f, 0.0f);
    ps.depth = 0;
    ps.specular = 0;
    ps.inside = 0;
    ps.nrcReady = 0;
}

__device__ __forceinline__ bool all_finite(v3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }

// Visibility of a shadow request as the reference decides it
// (pathtracerMdl.hlsl:57-74): no hit, or the first hit in depth-first order
// lies on a light's emitter instance.
__device__ __forceinline__ bool shadow_visible(const DevScene& s, int kind, v3 o, float tmax, v3 d)
{
    HitRec h;
    h.instId = SB_INVALID;
    uint32_t a = 0, b = 0;
    bool occl = trace_any_rec<false>(s, o, tmax, d, h, a, b);
    if (!occl) return true;
    if (kind == 1 && h.instId < s.numInstances && __ldg(&s.inst[h.instId].lightId) != -1) return true;
    return false;
}

// Adds a visible next-event contribution in the reference's order.
__device__ __forceinline__ void apply_shadow(v3& color, v3 cd, v3 cg)
{
    color = vadd(color, cd);
    color = vadd(color, cg);
}

// One iteration of the loop body of pathTraceCameraRays after closestHit
// (pathtracerMdl.hlsl:225-401).  Returns true when the path continues (the
// caller then increments depth and tests depth < maxDepth).  hit.primId holds
// the hit's compact leaf index: the triangle's world-space vertex data comes
// from the leaf's shading record (s.shadeRec, built by k_prep_shade with the
// arithmetic of pathtracerMdl.hlsl:237-267 applied to the instance, index
// and vertex buffers, so the values are the same bits).
__device__ __forceinline__ bool shade(const DevScene& s, const PathTracerParam& ubo, PathState& ps, bool found,
                                      const HitRec& hit, ShadowReq& sr, NrcShade* nq = nullptr)
{
    sr.kind = 0;
    if (!found) {
        // miss: the reference adds throughput * 0
        if (s.hasEnv) {
            int texel;
            v3 Le = env_lookup(s.env, ps.rd, texel);
            float misW = 1.0f;
            if (ps.depth > 0 && !ps.specular) {
                uint32_t total = ubo.numLights + 1u;
                float lpdf = env_pdf(s.env, texel, ps.rd) * (1.0f / (float)total);
                misW = ps.lastPdf / (ps.lastPdf + lpdf);
            }
            ps.color = vadd(ps.color, vscale(vmul(ps.throughput, Le), misW));
        } else {
            ps.color = vadd(ps.color, vmul(ps.throughput, V(0.0f, 0.0f, 0.0f)));
        }
        return false;
    }
    // The instance's ids and the leaf's shading record do not depend on each
    // other: all of them are requested before the light-id branch, so a
    // shaded hit waits for one round of loads instead of two.
    const InstanceConstants* ic = &s.inst[hit.instId];
    const int32_t lightId = __ldg(&ic->lightId);
    const int32_t materialId = __ldg(&ic->materialId);
    const uint32_t leaf = hit.primId;
    const bool recOk = leaf < s.numRec;
    float4 a0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), a1 = a0, a2 = a0, a3 = a0, a4 = a0, a5 = a0;
    if (recOk) {
        const float4* r = &s.shadeRec[6 * (size_t)leaf];
        a0 = __ldg(r);
        a1 = __ldg(r + 1);
        a2 = __ldg(r + 2);
        a3 = __ldg(r + 3);
        a4 = __ldg(r + 4);
        a5 = __ldg(r + 5);
    }
    if (lightId != -1 && (ps.depth == 0 || ps.specular)) {
        if ((uint32_t)lightId >= s.lightCapacity) { raise_status(s, STRELKA_DEV_LIGHT_OOB); return false; }
        const float4 lc = __ldg(&reinterpret_cast<const float4*>(&s.lights[lightId])[4]);  // color
        ps.color = vadd(ps.color, vmul(ps.throughput, V(lc.x, lc.y, lc.z)));
        return false;
    }
    if (lightId != -1) return false;  // diffuse bounce reached an emitter (reference reads mdlMaterials[-1])

    if (!recOk) {
        raise_status(s, STRELKA_DEV_NODE_OOB);
        return false;
    }
    const v3 p0 = xyz(a0), p1 = xyz(a1), p2 = xyz(a2);
    const v3 n0 = xyz(a3), n1 = xyz(a4), n2 = xyz(a5);
    const float uv0[2] = {a0.w, a1.w}, uv1[2] = {a2.w, a3.w}, uv2[2] = {a4.w, a5.w};
    v3 geomNormal = vnormalize(vcross(vsub(p1, p0), vsub(p2, p0)));
    const float bx = hit.u, by = hit.v;
    v3 worldPosition = interp3(p0, p1, p2, bx, by);
    v3 worldNormal = vnormalize(interp3(n0, n1, n2, bx, by));
    const float sign = ps.inside ? -1.0f : 1.0f;
    geomNormal = vscale(geomNormal, sign);
    worldNormal = vscale(worldNormal, sign);
    const float w = (1.0f - bx) - by;
    ShadeState st;
    st.u = (uv0[0] * w + uv1[0] * bx) + uv2[0] * by;
    st.v = (uv0[1] * w + uv1[1] * bx) + uv2[1] * by;
    if (ubo.debug == 1) {
        ps.color = V((worldNormal.x + 1.0f) * 0.5f, (worldNormal.y + 1.0f) * 0.5f, (worldNormal.z + 1.0f) * 0.5f);
        return false;
    }
    st.normal = worldNormal;
    st.geom_normal = geomNormal;
    st.position = worldPosition;
    Mat m;
    if (!load_material(s, materialId, st, m)) {
        raise_status(s, STRELKA_DEV_MATERIAL_OOB);
        return false;
    }
    if (nq) {
        nq->has = true;
        nq->pos = st.position;
        nq->normal = st.normal;
        nq->rough = m.fn == STRELKA_FN_LAMBERT ? 1.0f : m.roughness;
        if (nq->mode == 2 && ps.nrcReady) {
            nq->terminate = true;
            return false;
        }
    }
    const float ior1 = ps.inside ? -1.0f : 1.0f;  // BSDF_USE_MATERIAL_IOR = -1
    const float ior2 = ps.inside ? 1.0f : -1.0f;
    const v3 k1 = vneg(ps.rd);
    // EDF: intensity * edf with edf = 1
    ps.color = vadd(ps.color, vmul(vmul(ps.throughput, m.emission), V(1.0f, 1.0f, 1.0f)));

    // sampleLights (pathtracerMdl.hlsl:31-92; the environment is one extra light)
    const uint32_t numLights = ubo.numLights;
    const uint32_t total = numLights + (s.hasEnv ? 1u : 0u);
    if (total == 0) return false;  // reference: lightPdf = 0 * (1/0) = NaN, break
    const uint32_t lid = (uint32_t)((float)total * rand01(ps.rng));
    const float lightSelectionPdf = 1.0f / (float)total;
    v3 toLight = V(0.0f, 0.0f, 0.0f);
    float lightPdf = 0.0f;
    v3 Li = V(0.0f, 0.0f, 0.0f);
    float cs = 0.0f;
    int kind = 0;
    v3 so = V(0.0f, 0.0f, 0.0f);
    float stmax = 0.0f;
    if (lid >= numLights && s.hasEnv) {
        float r0 = rand01(ps.rng);
        float r1 = rand01(ps.rng);
        float pdf;
        v3 Le;
        v3 L = env_sample(s.env, r0, r1, pdf, Le);
        toLight = L;
        if (vdot(st.normal, L) > 0.0f && pdf > 0.0f && (Le.x != 0 || Le.y != 0 || Le.z != 0)) {
            kind = 2;
            so = offset_ray(st.position, st.geom_normal);
            stmax = 1e9f;
            lightPdf = pdf;
            Li = Le;
            cs = fsat(vdot(st.normal, L));
        }
    } else {
        if (lid >= s.lightCapacity) { raise_status(s, STRELKA_DEV_LIGHT_OOB); return false; }
        const UniformLight light = s.lights[lid];
        LightSample ls;
        ls.L = V(0.0f, 0.0f, 0.0f);
        ls.normal = V(0.0f, 0.0f, 0.0f);
        ls.pdf = 0.0f;
        ls.distToLight = 0.0f;
        if (light.type >= 0 && light.type <= 2) {
            float r0 = rand01(ps.rng);
            float r1 = rand01(ps.rng);
            ls = sample_light(light, st.position, r0, r1);
        }
        toLight = ls.L;
        v3 lc = V(light.color.x, light.color.y, light.color.z);
        if (vdot(st.normal, ls.L) > 0.0f && -vdot(ls.L, ls.normal) > 0.0f && (lc.x != 0 && lc.y != 0 && lc.z != 0)) {
            kind = 1;
            so = offset_ray(st.position, st.geom_normal);
            stmax = ls.distToLight;
            lightPdf = ls.pdf;
            Li = lc;
            cs = fsat(vdot(st.normal, ls.L));
        }
    }
    lightPdf *= lightSelectionPdf;

    // radiance = visibility * Li * saturate(dot(N, L)); evaluated for
    // visibility 1 here, the query is deferred when that is exact.
    bool inlineShadow = false;
    float vis = 1.0f;
    if (kind != 0 && !isfinite(Li.x + Li.y + Li.z)) {
        inlineShadow = true;
        vis = shadow_visible(s, kind, so, stmax, toLight) ? 1.0f : 0.0f;
    }
    v3 radiance = kind != 0 ? V(vis * Li.x * cs, vis * Li.y * cs, vis * Li.z * cs) : V(0.0f, 0.0f, 0.0f);
    if (vhasnan(radiance) || isnan(lightPdf)) return false;
    const bool nextEventValid = ((vdot(toLight, st.geom_normal) > 0.0f) != (ps.inside != 0)) && lightPdf != 0.0f;
    if (nextEventValid) {
        v3 radianceOverPdf = vdivs(radiance, lightPdf);
        EvalOut ev = bsdf_evaluate(m, st, k1, toLight, ior1, ior2);
        if (vhasnan(ev.bsdf_diffuse) || vhasnan(ev.bsdf_glossy)) return false;
        if (ev.pdf > 0.0f) {
            const float misWeight = (lightPdf == 0.0f) ? 1.0f : lightPdf / (lightPdf + ev.pdf);
            v3 wgt = vscale(vmul(ps.throughput, radianceOverPdf), misWeight);
            v3 cd = vmul(wgt, ev.bsdf_diffuse);
            v3 cg = vmul(wgt, ev.bsdf_glossy);
            if (kind == 0 || inlineShadow) {
                apply_shadow(ps.color, cd, cg);
            } else if (all_finite(ps.throughput) && isfinite(misWeight) && all_finite(ev.bsdf_diffuse) &&
                       all_finite(ev.bsdf_glossy)) {
                sr.kind = kind;
                sr.o = so;
                sr.tmax = stmax;
                sr.d = toLight;
                sr.cd = cd;
                sr.cg = cg;
            } else {
                // non-finite inputs: visibility 0 would not add +/-0, so query now
                if (shadow_visible(s, kind, so, stmax, toLight)) {
                    apply_shadow(ps.color, cd, cg);
                } else {
                    v3 r0 = V(0.0f * Li.x * cs, 0.0f * Li.y * cs, 0.0f * Li.z * cs);
                    if (vhasnan(r0)) return false;
                    v3 w0 = vscale(vmul(ps.throughput, vdivs(r0, lightPdf)), misWeight);
                    apply_shadow(ps.color, vmul(w0, ev.bsdf_diffuse), vmul(w0, ev.bsdf_glossy));
                }
            }
        }
    }

    float xi[4];
    xi[0] = rand01(ps.rng);
    xi[1] = rand01(ps.rng);
    xi[2] = rand01(ps.rng);
    xi[3] = rand01(ps.rng);
    SampleOut smp = bsdf_sample(m, st, k1, xi, ior1, ior2);
    if (smp.event == SB_EV_ABSORB) return false;
    ps.specular = (smp.event & SB_EV_SPECULAR) != 0;
    ps.inside = (smp.event & SB_EV_TRANSMISSION) != 0;
    const v3 rayOriginNext = offset_ray(st.position, vscale(st.geom_normal, ps.inside ? -1.0f : 1.0f));
    ps.throughput = vmul(ps.throughput, smp.bsdf_over_pdf);
    ps.lastPdf = smp.pdf;
    if (nq && (m.fn == STRELKA_FN_LAMBERT || m.roughness >= nq->diffuseRoughness)) ps.nrcReady = 1;
    if (ps.depth > 3) {
        float p = fmaxf(ps.throughput.x, fmaxf(ps.throughput.y, ps.throughput.z));
        if (rand01(ps.rng) > p) return false;
        float sc = 1.0f / (p + 1e-5f);
        ps.throughput = vscale(ps.throughput, sc);
    }
    ps.ro = rayOriginNext;
    ps.tmax = 1e9f;
    ps.rd = smp.k2;
    return true;
}

}  // namespace sb
