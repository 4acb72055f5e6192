"""The path tracer's estimators against expectations computed independently
(CPU, the oracle's path tracer; the GPU kernels equal it bit for bit):
the environment light under Lambert, GGX conductor and rough dielectric
quads (quadrature), and a white furnace (closed form).

Environment scenes: one large Lambert quad of albedo a facing +y, lit only by a seeded
piecewise-constant environment (64 x 32 texels, random radiance plus a bright
patch), seen from above; maxDepth 2.  Every sample takes the path of
pathTraceCameraRays (shaders/pathtracerMdl.hlsl:204-404) for one hit: a
next-event sample of the environment and a cosine-sampled bounce that escapes
to it, combined by the balance heuristic.  Nothing else is in the scene, so
each sample is an independent estimate of

    E = integral over the upper hemisphere of
        a/pi * Le(w) * (c^2 p_L(w) + c p_B(w)) / (p_L(w) + p_B(w)) dw,

c = cos(theta), p_B = (c + 1e-6)/pi (the sampled Lambert's pdf), p_L the
environment's pdf (rows by the marginal CDF, columns by the row's CDF, over
the texel's solid angle at sin(theta)).  The c^2 of the next-event term is
the reference's: its radiance carries saturate(dot(N, L))
(pathtracerMdl.hlsl:31-92) and the BSDF evaluation its own cosine.  The
quadrature uses only the CDF tables and the texel radiances, not the
sampler, so a sampler whose directions do not follow the pdf it reports, or
a wrong MIS weight, moves the mean off E by many standard errors."""
import ctypes as C

import numpy as np

import oracle
from strelka_b200 import abi, scenes

A = 0.7          # albedo
EW, EH = 64, 32  # environment texels


def _pack(fn, v):
    arr = (C.c_float * len(v))(*v)
    return getattr(abi.load(), fn)(arr)


def _environment(seed):
    rng = np.random.default_rng(seed)
    env = np.zeros((EH, EW, 4), np.float32)
    env[..., :3] = rng.uniform(0.05, 1.0, (EH, EW, 3)).astype(np.float32)
    env[4:7, 20:24, :3] *= 40.0  # a bright patch above the horizon
    env[..., 3] = 1.0
    marg = np.zeros(EH + 1, np.float32)
    cond = np.zeros(EH * (EW + 1), np.float32)
    integral = C.c_float(0.0)
    lib = abi.load()
    assert lib.strelka_envmap_build_cdf_host(env.ctypes.data, EW, EH, marg.ctypes.data, cond.ctypes.data,
                                             C.byref(integral)) == abi.OK
    return env, marg, cond, float(integral.value)


def _scene(seed, fn=abi.FN_LAMBERT, base=(A, A, A), roughness=1.0, environment=None):
    S = 1000.0
    pos = np.array([[-S, 0, -S], [-S, 0, S], [S, 0, S], [S, 0, -S]], np.float32)
    vb = (abi.Vertex * 4)()
    for i in range(4):
        vb[i].position[:] = pos[i]
        vb[i].normal = _pack("strelka_pack_normal", [0.0, 1.0, 0.0])
        vb[i].tangent = _pack("strelka_pack_normal", [1.0, 0.0, 0.0])
        vb[i].uv = _pack("strelka_pack_uv", [0.0, 0.0])
    ib = np.array([0, 1, 2, 0, 2, 3], np.uint32)
    inst = abi.InstanceConstants()
    for m in (inst.objectToWorld, inst.worldToObject, inst.normalMatrix):
        for k in range(4):
            m.m[5 * k] = 1.0
    inst.materialId, inst.indexOffset, inst.indexCount, inst.lightId = 0, 0, 6, -1
    mat = abi.MdlMaterial(0, 0, fn, 0)
    args = np.zeros(12, np.float32)  # StrelkaMaterialArgs
    args[0:3] = base
    args[3] = roughness
    args[7] = 1.5   # ior
    tri = pos[ib].reshape(-1, 3)
    nodes = scenes.bvh_build(tri, np.zeros(6, np.uint32), np.repeat(np.arange(2, dtype=np.uint32), 3))
    env, marg, cond, integral = environment if environment is not None else _environment(seed)
    hs = scenes.HostScene(
        vb=np.frombuffer(bytes(vb), np.uint8).copy(), ib=ib,
        instances=np.frombuffer(bytes(inst), np.uint8).copy(),
        lights=np.zeros(112, np.uint8), num_lights=0,
        materials=np.frombuffer(bytes(mat), np.uint8).copy(),
        arg_block=args.view(np.uint8).copy(), resource_infos=np.zeros(16, np.uint8), textures=[],
        env=env, env_marginal=marg, env_conditional=cond, env_integral=integral,
        nodes=nodes, num_triangles=2, camera=abi.PathTracerParam())
    return hs


def _expectation(hs, sub=64):
    """The integral above by the midpoint rule over each texel's rows (Le and
    p_L do not vary with phi inside a texel)."""
    env, marg, cond = hs.env, hs.env_marginal, hs.env_conditional.reshape(EH, EW + 1)
    dphi = 2.0 * np.pi / EW
    total = np.zeros(3)
    for y in range(EH // 2):  # theta < pi/2
        t = (y + (np.arange(sub) + 0.5) / sub) * np.pi / EH
        dth = np.pi / EH / sub
        c, s = np.cos(t), np.sin(t)
        p_row = float(marg[y + 1]) - float(marg[y])
        for x in range(EW):
            p_col = float(cond[y, x + 1]) - float(cond[y, x])
            p_l = p_row * p_col / ((2.0 * np.pi / EW) * (np.pi / EH) * s)
            p_b = (c + 1e-6) / np.pi
            w = (c * c * p_l + c * p_b) / (p_l + p_b)
            total += env[y, x, :3].astype(np.float64) * (A / np.pi) * np.sum(w * s) * dth * dphi
    return total


def test_environment_estimator_matches_its_expectation():
    hs = _scene(seed=3)
    W = H = 64
    spp = 32
    p = hs.look_at(W, H, eye=(0.0, 10.0, 4.0), target=(0.0, 0.0, 0.0), fov_deg=40.0, spp=spp, maxDepth=2,
                   numLights=0, frameNumber=1, stratifiedSamplingType=1)
    samples = oracle.pathtrace(oracle.SceneView(hs), p).astype(np.float64).reshape(-1, 3)
    n = samples.shape[0]
    assert n == W * H * spp and np.isfinite(samples).all()
    mean = samples.mean(0)
    se = samples.std(0) / np.sqrt(n)
    expect = _expectation(hs)
    # 5 standard errors, plus 1e-4 relative for the 1e-6 in p_B and rounding
    assert np.all(np.abs(mean - expect) <= 5.0 * se + 1e-4 * expect), (mean, expect, se)
    # and the bound is tight enough to matter: a few percent of the value
    assert np.all(5.0 * se < 0.03 * expect), (se, expect)


def _ggx_expectation(hs, k1, f0, roughness, sub=12):
    """The GGX conductor's counterpart: next-event and sampled-reflection
    terms of pathTraceCameraRays with the native conductor (D, Smith G from
    G1, Schlick F; sampled half vectors with pdf D (n.h), reflected, so the
    reported pdf D (n.h) / (4 v.h) is the density of the direction):

        E = integral over n.l > 0 of Le f(v, l) (n.l) ((n.l) p_L + p_B) / (p_L + p_B) dl,
        f = F D G / (4 (n.v)(n.l)).

    Midpoint rule over sub x sub cells of every texel above the horizon."""
    env, marg, cond = hs.env, hs.env_marginal, hs.env_conditional.reshape(EH, EW + 1)
    alpha = max(roughness * roughness, 1e-3)
    a2 = alpha * alpha
    f0 = np.asarray(f0, np.float64)
    nov = k1[1]

    def g1(x):
        return 2.0 * x / (x + np.sqrt(a2 + (1.0 - a2) * x * x))

    total = np.zeros(3)
    j = (np.arange(sub) + 0.5) / sub
    for y in range(EH // 2):
        t = (y + j[:, None]) * np.pi / EH                       # (sub, 1)
        p_row = float(marg[y + 1]) - float(marg[y])
        for x in range(EW):
            ph = ((x + j[None, :]) / EW - 0.5) * 2.0 * np.pi     # (1, sub)
            st, ct = np.sin(t), np.cos(t)
            lx, ly, lz = st * np.sin(ph), ct + 0.0 * ph, -st * np.cos(ph)
            hx, hy, hz = lx + k1[0], ly + k1[1], lz + k1[2]
            hn = np.sqrt(hx * hx + hy * hy + hz * hz)
            noh = np.clip(hy / hn, 0.0, 1.0)
            voh = np.clip((hx * k1[0] + hy * k1[1] + hz * k1[2]) / hn, 0.0, 1.0)
            nol = ly
            tt = noh * noh * (a2 - 1.0) + 1.0
            D = a2 / (np.pi * tt * tt)
            G = g1(nov) * g1(nol)
            w5 = np.clip(1.0 - voh, 0.0, 1.0) ** 5
            p_col = float(cond[y, x + 1]) - float(cond[y, x])
            p_l = p_row * p_col / ((2.0 * np.pi / EW) * (np.pi / EH) * st)
            p_b = D * noh / (4.0 * voh)
            common = D * G / (4.0 * nov) * (nol * p_l + p_b) / (p_l + p_b)  # f (n.l) without F, times the weights
            dw = st * (np.pi / EH / sub) * (2.0 * np.pi / EW / sub)
            for c in range(3):
                F = f0[c] + (1.0 - f0[c]) * w5
                total[c] += env[y, x, c] * np.sum(F * common * dw)
    return total


def test_ggx_conductor_estimator_matches_its_expectation():
    # the native GGX conductor (parity against MDL is unpinned by
    # construction): a far camera with a 0.5-degree field of view, so every
    # sample sees the quad from nearly one direction v
    f0, rough = (0.9, 0.6, 0.3), 0.6
    hs = _scene(seed=5, fn=abi.FN_GGX_CONDUCTOR, base=f0, roughness=rough)
    eye = np.array([0.0, 600.0, 800.0])
    W = H = 64
    spp = 32
    p = hs.look_at(W, H, eye=tuple(eye), target=(0.0, 0.0, 0.0), fov_deg=0.5, spp=spp, maxDepth=2,
                   numLights=0, frameNumber=2, stratifiedSamplingType=1)
    samples = oracle.pathtrace(oracle.SceneView(hs), p).astype(np.float64).reshape(-1, 3)
    n = samples.shape[0]
    assert np.isfinite(samples).all()
    mean = samples.mean(0)
    se = samples.std(0) / np.sqrt(n)
    expect = _ggx_expectation(hs, eye / np.linalg.norm(eye), f0, rough)
    assert np.all(np.abs(mean - expect) <= 5.0 * se + 2e-3 * expect), (mean, expect, se)
    assert np.all(5.0 * se < 0.05 * expect), (se, expect)


def _fresnel_dielectric(c, eta):
    sin2t = eta * eta * (1.0 - c * c)
    cost = np.sqrt(np.clip(1.0 - sin2t, 0.0, 1.0))
    rs = (c - eta * cost) / (c + eta * cost)
    rp = (eta * c - cost) / (eta * c + cost)
    return np.where(sin2t >= 1.0, 1.0, 0.5 * (rs * rs + rp * rp))


def _env_texel_pdf(hs, d):
    """Le and p_L of directions d (..., 3) as the miss and env_pdf read them."""
    env, marg, cond = hs.env, hs.env_marginal, hs.env_conditional.reshape(EH, EW + 1)
    u = np.arctan2(d[..., 0], -d[..., 2]) / (2.0 * np.pi) + 0.5
    v = np.arccos(np.clip(d[..., 1], -1.0, 1.0)) / np.pi
    x = np.clip((u * EW).astype(int), 0, EW - 1)
    y = np.clip((v * EH).astype(int), 0, EH - 1)
    st = np.sqrt(np.clip(1.0 - d[..., 1] ** 2, 0.0, 1.0))
    p_l = ((marg[y + 1].astype(np.float64) - marg[y]) * (cond[y, x + 1].astype(np.float64) - cond[y, x])
           / ((2.0 * np.pi / EW) * (np.pi / EH) * st))
    return env[y, x, :3].astype(np.float64), p_l


def _dielectric_expectation(hs, k1, tint, roughness, ior, n_theta=384, n_phi=768):
    """The rough dielectric seen from outside (eta = 1 / ior):
    reflection as the conductor with the dielectric's Fresnel and no tint
    (evaluation and next-event sampling cover it), plus the transmitted
    half: a half vector h drawn with pdf D (n.h), kept with probability
    1 - F(v.h), the direction refracted through h (absorbed unless it goes
    below the surface), weight tint G (v.h) / ((n.v)(n.h)), and the
    environment below reached with the MIS weight of the pdf the sampler
    reports, (1 - F) D (n.h), against p_L.  Both by the midpoint rule over
    the half-vector hemisphere: E = sum over h of pdf(h) x value."""
    alpha = max(roughness * roughness, 1e-3)
    a2 = alpha * alpha
    eta = 1.0 / ior
    nov = k1[1]

    def g1(x):
        return 2.0 * x / (x + np.sqrt(a2 + (1.0 - a2) * x * x))

    th = (np.arange(n_theta) + 0.5) / n_theta * (np.pi / 2)
    ph = (np.arange(n_phi) + 0.5) / n_phi * (2.0 * np.pi)
    T, P = np.meshgrid(th, ph, indexing="ij")
    h = np.stack([np.sin(T) * np.cos(P), np.cos(T), np.sin(T) * np.sin(P)], -1)
    dh = np.sin(T) * (np.pi / 2 / n_theta) * (2.0 * np.pi / n_phi)
    noh = h[..., 1]
    voh = h @ k1
    tt = noh * noh * (a2 - 1.0) + 1.0
    D = a2 / (np.pi * tt * tt)
    pdf_h = D * noh * dh                         # probability of each cell
    ok = voh > 0.0
    F = _fresnel_dielectric(np.where(ok, voh, 1.0), eta)
    total = np.zeros(3)
    # reflection: k2 = 2 (v.h) h - v, kept when n.k2 > 0
    k2 = 2.0 * voh[..., None] * h - k1
    nol = k2[..., 1]
    keep = ok & (nol > 0.0)
    le, p_l = _env_texel_pdf(hs, k2)
    G = g1(nov) * g1(np.where(keep, nol, 1.0))
    w_b = G * voh / (nov * noh)                  # bsdf over pdf (F cancels the choice)
    p_b = F * D * noh / (4.0 * np.where(ok, voh, 1.0))
    bsdf_part = np.where(keep, F * w_b * p_b / (p_b + p_l), 0.0)          # sampled reflections
    # next-event part, written over the same cells: f cos x cos x p_L / (p_L + p_B) per unit
    # direction, and a direction cell is a half-vector cell times 4 (v.h)
    nee_part = np.where(keep, F * D * G / (4.0 * nov) * nol * p_l / (p_l + p_b) * 4.0 * voh * dh, 0.0)
    for c in range(3):
        total[c] += np.sum(pdf_h * bsdf_part * le[..., c]) + np.sum(nee_part * le[..., c])
    # transmission: refraction through h, kept when n.k2 < 0
    sin2t = eta * eta * (1.0 - voh * voh)
    c2 = np.sqrt(np.clip(1.0 - sin2t, 0.0, 1.0))
    sc = eta * voh - c2
    k2 = -eta * k1 + sc[..., None] * h
    k2 = k2 / np.linalg.norm(k2, axis=-1, keepdims=True)
    nol = k2[..., 1]
    keep = ok & (nol < 0.0) & (sin2t < 1.0)
    le, p_l = _env_texel_pdf(hs, k2)
    G = g1(nov) * g1(np.where(keep, -nol, 1.0))
    w_t = G * voh / (nov * noh)
    p_rep = (1.0 - F) * D * noh
    trans = np.where(keep, (1.0 - F) * w_t * p_rep / (p_rep + p_l), 0.0)
    for c in range(3):
        total[c] += np.sum(pdf_h * trans * tint[c] * le[..., c])
    return total


def test_ggx_dielectric_estimator_matches_its_expectation():
    # the native rough dielectric from outside: reflected and transmitted
    # halves, the latter escaping below the quad to the environment
    tint, rough, ior = (0.9, 0.8, 0.7), 0.6, 1.5
    hs = _scene(seed=6, fn=abi.FN_GGX_DIELECTRIC, base=tint, roughness=rough)
    eye = np.array([0.0, 600.0, 800.0])
    p = hs.look_at(64, 64, eye=tuple(eye), target=(0.0, 0.0, 0.0), fov_deg=0.5, spp=32, maxDepth=2,
                   numLights=0, frameNumber=3, stratifiedSamplingType=1)
    samples = oracle.pathtrace(oracle.SceneView(hs), p).astype(np.float64).reshape(-1, 3)
    assert np.isfinite(samples).all()
    mean = samples.mean(0)
    se = samples.std(0) / np.sqrt(samples.shape[0])
    expect = _dielectric_expectation(hs, eye / np.linalg.norm(eye), tint, rough, ior)
    assert np.all(np.abs(mean - expect) <= 5.0 * se + 2e-3 * expect), (mean, expect, se)
    assert np.all(5.0 * se < 0.05 * expect), (se, expect)


def _lambert_expectation(hs, sub=16):
    """_expectation for an environment of any size, vectorised over columns."""
    env = hs.env
    eh, ew = env.shape[:2]
    marg = hs.env_marginal.astype(np.float64)
    cond = hs.env_conditional.reshape(eh, ew + 1).astype(np.float64)
    p_col = cond[:, 1:] - cond[:, :-1]
    dth, dphi = np.pi / eh / sub, 2.0 * np.pi / ew
    total = np.zeros(3)
    for y in range(eh // 2):
        t = (y + (np.arange(sub) + 0.5) / sub) * np.pi / eh
        c, s = np.cos(t), np.sin(t)
        p_l = (marg[y + 1] - marg[y]) * p_col[y][:, None] / ((2.0 * np.pi / ew) * (np.pi / eh) * s[None, :])
        p_b = (c + 1e-6) / np.pi
        w = (c * c * p_l + c * p_b) / (p_l + p_b)
        total += env[y, :, :3].astype(np.float64).T @ (w * s[None, :]).sum(1) * (A / np.pi) * dth * dphi
    return total


def test_environment_estimator_on_the_workload_environment():
    # the large render's own 1024 x 512 environment with its sun lobe (the
    # bench frame's only light), under the same Lambert quad
    big = scenes.large(width=8, height=8, instances=1, frequency=2, num_textures=1, tex_size=16, env_width=1024,
                       env_height=512, max_depth=2, spp=1, seed=0)
    environment = (big.env, big.env_marginal, big.env_conditional, big.env_integral)
    hs = _scene(seed=0, environment=environment)
    p = hs.look_at(64, 64, eye=(0.0, 10.0, 4.0), target=(0.0, 0.0, 0.0), fov_deg=40.0, spp=32, maxDepth=2,
                   numLights=0, frameNumber=7, stratifiedSamplingType=1)
    samples = oracle.pathtrace(oracle.SceneView(hs), p).astype(np.float64).reshape(-1, 3)
    assert np.isfinite(samples).all()
    mean = samples.mean(0)
    se = samples.std(0) / np.sqrt(samples.shape[0])
    expect = _lambert_expectation(hs)
    small = _scene(seed=3)
    assert np.allclose(_lambert_expectation(small, sub=64), _expectation(small, sub=64), rtol=1e-9)
    assert np.all(np.abs(mean - expect) <= 5.0 * se + 1e-4 * expect), (mean, expect, se)
    assert np.all(5.0 * se < 0.03 * expect), (se, expect)


def _furnace(albedo, le):
    """A closed box [-1, 1]^3 seen from inside: 12 inward-facing Lambert
    triangles of the given albedo that also emit le, and a black environment
    (present, so the loop of pathTraceCameraRays goes on past the first hit,
    but contributing nothing)."""
    faces = []
    for axis in range(3):
        for side in (-1.0, 1.0):
            n = np.zeros(3)
            n[axis] = -side                      # inward
            u, v = [a for a in range(3) if a != axis]
            quad = []
            for cu, cv in ((-1, -1), (-1, 1), (1, 1), (1, -1)):
                p = np.zeros(3)
                p[axis], p[u], p[v] = side, cu, cv
                quad.append(p)
            for tri in ((0, 1, 2), (0, 2, 3)):
                a, b, c = (quad[i] for i in tri)
                if np.dot(np.cross(b - a, c - a), n) < 0:
                    b, c = c, b
                faces.append((a, b, c, n))
    nv = 3 * len(faces)
    vb = (abi.Vertex * nv)()
    pos = np.zeros((nv, 3), np.float32)
    for f, (a, b, c, n) in enumerate(faces):
        for k, p in enumerate((a, b, c)):
            i = 3 * f + k
            pos[i] = p
            vb[i].position[:] = p
            vb[i].normal = _pack("strelka_pack_normal", list(n))
            vb[i].tangent = _pack("strelka_pack_normal", list(np.roll(n, 1)))
            vb[i].uv = _pack("strelka_pack_uv", [0.0, 0.0])
    ib = np.arange(nv, dtype=np.uint32)
    inst = abi.InstanceConstants()
    for m in (inst.objectToWorld, inst.worldToObject, inst.normalMatrix):
        for k in range(4):
            m.m[5 * k] = 1.0
    inst.materialId, inst.indexOffset, inst.indexCount, inst.lightId = 0, 0, nv, -1
    mat = abi.MdlMaterial(0, 0, abi.FN_LAMBERT, 0)
    args = np.zeros(12, np.float32)
    args[0:3] = albedo
    args[3] = 1.0
    args[4:7] = le
    args[7] = 1.5
    prim = np.repeat(np.arange(len(faces), dtype=np.uint32), 3)
    nodes = scenes.bvh_build(pos, np.zeros(nv, np.uint32), prim)
    env = np.zeros((4, 8, 4), np.float32)
    marg = np.zeros(5, np.float32)
    cond = np.zeros(4 * 9, np.float32)
    integral = C.c_float(0.0)
    assert abi.load().strelka_envmap_build_cdf_host(env.ctypes.data, 8, 4, marg.ctypes.data, cond.ctypes.data,
                                                    C.byref(integral)) == abi.OK
    return scenes.HostScene(
        vb=np.frombuffer(bytes(vb), np.uint8).copy(), ib=ib, instances=np.frombuffer(bytes(inst), np.uint8).copy(),
        lights=np.zeros(112, np.uint8), num_lights=0, materials=np.frombuffer(bytes(mat), np.uint8).copy(),
        arg_block=args.view(np.uint8).copy(), resource_infos=np.zeros(16, np.uint8), textures=[],
        env=env, env_marginal=marg, env_conditional=cond, env_integral=float(integral.value),
        nodes=nodes, num_triangles=len(faces), camera=abi.PathTracerParam())


def test_white_furnace():
    # every hit adds throughput * Le and every bounce multiplies the
    # throughput by the albedo, so a path of maxDepth hits carries
    # Le (1 - a^D) / (1 - a).  Without Russian roulette (D <= 4) that is
    # every sample's value; with it (depth > 3, survival max(throughput),
    # reweighted by 1 / (p + 1e-5)) it is the mean
    albedo, le = (0.5, 0.7, 0.9), (1.0, 2.0, 0.5)
    hs = _furnace(albedo, le)
    view = oracle.SceneView(hs)
    a, e = np.array(albedo), np.array(le)
    for depth, spp in ((4, 4), (12, 32)):
        p = hs.look_at(64, 64, eye=(0.1, 0.05, -0.2), target=(0.3, -0.2, 1.0), fov_deg=100.0, spp=spp,
                       maxDepth=depth, numLights=0, frameNumber=depth, stratifiedSamplingType=1)
        s = oracle.pathtrace(view, p).astype(np.float64).reshape(-1, 3)
        expect = e * (1.0 - a ** depth) / (1.0 - a)
        assert np.isfinite(s).all()
        if depth <= 4:
            assert np.allclose(s, expect, rtol=1e-5, atol=0.0), np.abs(s - expect).max(0)
        else:
            mean, se = s.mean(0), s.std(0) / np.sqrt(s.shape[0])
            assert np.all(np.abs(mean - expect) <= 5.0 * se + 1e-4 * expect), (mean, expect, se)
            assert np.all(5.0 * se < 0.02 * expect), (se, expect)
