"""Reduction, accumulation and tonemap passes on the GPU against the oracle,
bit for bit; the fused resolve equals the three passes in sequence."""
import numpy as np
import pytest

import oracle
from strelka_b200 import abi
from strelka_b200.render import (Accumulation, ReductionPass, Tonemap, accumulation_param, ptr, resolve,
                                 tonemap_param, to_device)

pytestmark = pytest.mark.gpu

W, H, SPP = 37, 23, 5


def dev(torch, a):
    return to_device(np.ascontiguousarray(a, np.float32)).view(torch.float32)


def host(t):
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def data(cuda):
    rng = np.random.default_rng(0)
    sb = (rng.gamma(0.5, 1.0, W * H * SPP * 3)).astype(np.float32)
    sb[::97] = 0.0
    hist = np.concatenate([rng.uniform(0, 3, (W * H, 3)), np.ones((W * H, 1))], 1).astype(np.float32).ravel()
    p = abi.PathTracerParam()
    p.dimension[0], p.dimension[1], p.spp = W, H, SPP
    return sb, hist, p


def test_reduction(cuda, data):
    sb, _, p = data
    out = cuda.zeros(W * H * 4, dtype=cuda.float32, device="cuda")
    d = abi.ReductionDesc(p, ptr(dev(cuda, sb)), ptr(out))
    sbd = dev(cuda, sb)
    d.sampleBuffer = ptr(sbd)
    ReductionPass().execute(d, W * H, 1, 0)
    assert np.array_equal(host(out).view(np.uint32), oracle.reduce(p, sb).view(np.uint32))


@pytest.mark.parametrize("iteration", [0, 1, 7, 1000])
def test_accumulation(cuda, data, iteration):
    sb, hist, p = data
    cur = oracle.reduce(p, sb)
    ap = accumulation_param(W, H, iteration)
    out = cuda.zeros(W * H * 4, dtype=cuda.float32, device="cuda")
    a, b = dev(cuda, cur), dev(cuda, hist)
    Accumulation().execute(abi.AccumulationDesc(ap, ptr(a), ptr(b), ptr(out)), W, H, 0)
    assert np.array_equal(host(out).view(np.uint32), oracle.accumulate(ap, cur, hist).view(np.uint32))


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_tonemap(cuda, data, kind):
    sb, _, p = data
    img = oracle.reduce(p, sb)
    tp = tonemap_param(W, H, kind)
    out = cuda.zeros(W * H * 4, dtype=cuda.float32, device="cuda")
    a = dev(cuda, img)
    Tonemap().execute(abi.TonemapDesc(tp, ptr(a), ptr(out)), W, H, 0)
    ref = oracle.tonemap(tp, img)
    g = host(out)
    both_nan = np.isnan(g) & np.isnan(ref)
    assert np.array_equal(g.view(np.uint32)[~both_nan], ref.view(np.uint32)[~both_nan])
    assert np.array_equal(np.isnan(g), np.isnan(ref))


@pytest.mark.parametrize("accumulate", [False, True])
def test_resolve_equals_sequence(cuda, data, accumulate):
    sb, hist, p = data
    tp = tonemap_param(W, H, 1)
    ap = accumulation_param(W, H, 3)
    cur = oracle.reduce(p, sb)
    acc = oracle.accumulate(ap, cur, hist) if accumulate else cur
    tm = oracle.tonemap(tp, acc)
    sbd, hd = dev(cuda, sb), dev(cuda, hist)
    acc_out = cuda.zeros(W * H * 4, dtype=cuda.float32, device="cuda")
    tm_out = cuda.zeros(W * H * 4, dtype=cuda.float32, device="cuda")
    rgba8 = cuda.zeros(W * H * 4, dtype=cuda.uint8, device="cuda")
    resolve(p, sbd, tp, ap if accumulate else None, hd if accumulate else None, acc_out, tm_out, rgba8)
    assert np.array_equal(host(acc_out).view(np.uint32), acc.view(np.uint32))
    assert np.array_equal(host(tm_out).view(np.uint32), tm.view(np.uint32))
    q = (np.clip(tm, 0, 1) * np.float32(255) + np.float32(0.5)).astype(np.int32).astype(np.uint8)
    q[3::4] = 255
    assert np.array_equal(host(rgba8), q)


def test_bad_arguments(cuda, data):
    sb, _, p = data
    out = cuda.zeros(W * H * 4, dtype=cuda.float32, device="cuda")
    sbd = dev(cuda, sb)
    d = abi.ReductionDesc(p, ptr(sbd), ptr(out))
    with pytest.raises(abi.StrelkaError) as e:
        ReductionPass().execute(d, W * H + 1, 1, 0)
    assert e.value.code == abi.ERR_INVALID_ARGUMENT


# upscale pass (upscalepass.hlsl:9-21) and the fused tonemap + upscale + 8-bit blit
UPSCALE_SIZES = [(37, 23, 74, 46), (37, 23, 1920 // 20, 1080 // 20), (64, 32, 64, 32), (40, 30, 17, 11)]


@pytest.mark.parametrize("sizes", UPSCALE_SIZES)
def test_upscale(cuda, sizes):
    from strelka_b200.render import UpscalePass, upscale_param

    iw, ih, ow, oh = sizes
    rng = np.random.default_rng(iw * 7 + ow)
    img = np.concatenate([rng.gamma(0.7, 1.0, (iw * ih, 3)), np.ones((iw * ih, 1))], 1).astype(np.float32).ravel()
    src = dev(cuda, img)
    out = cuda.full((ow * oh * 4,), -1.0, dtype=cuda.float32, device="cuda")
    up = upscale_param(ow, oh)
    UpscalePass().execute(abi.UpscaleDesc(up, ptr(src), iw, ih, ptr(out)), ow, oh, 0)
    cuda.cuda.synchronize()
    assert np.array_equal(host(out).view(np.uint32), oracle.upscale(up, img, iw, ih).view(np.uint32))


@pytest.mark.parametrize("kind", [0, 1, 2])
@pytest.mark.parametrize("sizes", UPSCALE_SIZES[:2])
def test_tonemap_upscale_equals_sequence(cuda, kind, sizes):
    from strelka_b200.render import tonemap_upscale, upscale_param

    iw, ih, ow, oh = sizes
    rng = np.random.default_rng(kind + iw)
    img = np.concatenate([rng.gamma(0.7, 1.0, (iw * ih, 3)), np.ones((iw * ih, 1))], 1).astype(np.float32).ravel()
    tp = tonemap_param(iw, ih, kind)
    up = upscale_param(ow, oh)
    expect = oracle.upscale(up, oracle.tonemap(tp, img), iw, ih)
    out = cuda.zeros(ow * oh * 4, dtype=cuda.float32, device="cuda")
    out8 = cuda.zeros(ow * oh * 4, dtype=cuda.uint8, device="cuda")
    tonemap_upscale(tp, dev(cuda, img), up, out, out8)
    cuda.cuda.synchronize()
    got = host(out)
    assert np.array_equal(got.view(np.uint32), expect.view(np.uint32))
    q = np.clip(expect.reshape(-1, 4)[:, :3], 0, 1) * np.float32(255) + np.float32(0.5)
    assert np.array_equal(host(out8).reshape(-1, 4)[:, :3], q.astype(np.int32).astype(np.uint8))
    assert (host(out8).reshape(-1, 4)[:, 3] == 255).all()


def test_upscale_bad_arguments(cuda):
    from strelka_b200.render import UpscalePass, tonemap_upscale, upscale_param

    buf = cuda.zeros(64, dtype=cuda.float32, device="cuda")
    up = upscale_param(4, 4)
    with pytest.raises(abi.StrelkaError):
        UpscalePass().execute(abi.UpscaleDesc(up, ptr(buf), 4, 4, ptr(buf)), 5, 4, 0)  # w != dimension
    with pytest.raises(abi.StrelkaError):
        UpscalePass().execute(abi.UpscaleDesc(up, ptr(buf), 0, 4, ptr(buf)), 4, 4, 0)
    with pytest.raises(abi.StrelkaError):
        tonemap_upscale(tonemap_param(4, 4, 9), buf, up, buf)  # unknown tonemapper


def test_mdl_readers_match_oracle(cuda):
    rng = np.random.default_rng(11)
    buf = rng.integers(0, 256, 4096, dtype=np.uint8)
    buf[rng.integers(0, 4096, 500)] = 0  # zero bytes for the bool reader
    n = 20000
    offs = rng.integers(0, 4200, n).astype(np.uint32)  # unaligned and past the end too
    kinds = rng.integers(0, 5, n).astype(np.uint32)
    expect = oracle.mdl_read(buf, offs, kinds)
    out = cuda.zeros(n, dtype=cuda.int64, device="cuda")
    b = to_device(buf)
    o, k = to_device(offs), to_device(kinds)
    abi.check(abi.load().strelka_mdl_read(ptr(b), buf.size, ptr(o), ptr(k), n, ptr(out), None))
    cuda.cuda.synchronize()
    assert np.array_equal(host(out).view(np.uint64), expect)
