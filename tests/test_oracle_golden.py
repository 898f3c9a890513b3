"""The oracle against the reference's own fixtures.

Pins: the rest-density golden vector (scripts/rest_density.csv), the radix
known-answer tests of sorter.rs:585-646, and the radix mirror
`cpu_radix_sort` (sorter.rs:465-559) against the stable-sort definition.
"""
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN
from fluid_step import _abi, scene

SENT = 0xFFFFFFFF


def padded(hashes):
    """padded_entries (sorter.rs:561-579): index = position, pad with sentinels."""
    h = np.asarray(hashes, dtype=np.uint32)
    n = len(h)
    t = 1 << max(0, (n - 1).bit_length())
    k = np.full(t, SENT, np.uint32)
    v = np.full(t, SENT, np.uint32)
    k[:n] = h
    v[:n] = np.arange(n, dtype=np.uint32)
    return k, v


def kat_inputs():
    i = np.arange(1000, dtype=np.uint64)
    mult = ((i * 2654435761 + (i >> 3)) & 0xFFFFFFFF) % 131072
    return {
        "sort_small_known": [3, 1, 4, 1, 5, 9, 2, 6],
        "sort_matches_stdlib": mult.astype(np.uint32),
        "sort_all_same_hash": [42] * 300,
        "sort_reverse_order": list(range(511, -1, -1)),
        "sentinels_land_at_end": list(range(100)),
    }


def stable_reference(k, v):
    order = np.argsort(k, kind="stable")
    return k[order], v[order]


@pytest.mark.parametrize("name", list(kat_inputs()))
@pytest.mark.parametrize("algo", ["mirror", "parallel", "bitonic"])
def test_sort_known_answers(oracle_mod, name, algo):
    k, v = padded(kat_inputs()[name])
    fn = {"mirror": oracle_mod.sort_radix_mirror, "parallel": oracle_mod.sort_radix_parallel,
          "bitonic": oracle_mod.sort_bitonic}[algo]
    ks, vs = fn(k, v)
    assert np.all(ks[:-1] <= ks[1:]), "not sorted"
    assert np.array_equal(ks, np.sort(k))                       # sort_matches_stdlib
    if name == "sentinels_land_at_end":
        assert int(np.searchsorted(ks, SENT)) == 100
    # the pairs are a permutation of the input pairs
    assert np.array_equal(np.sort(ks.astype(np.uint64) << 32 | vs),
                          np.sort(k.astype(np.uint64) << 32 | v))
    if algo != "bitonic":                                       # radix is stable
        rk, rv = stable_reference(k, v)
        assert np.array_equal(vs, rv)


def test_radix_mirror_random(oracle_mod):
    rng = np.random.default_rng(7)
    for n in (1, 2, 255, 2049, 5000, 1 << 14):
        k = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        v = np.arange(n, dtype=np.uint32)
        a = oracle_mod.sort_radix_mirror(k, v)
        b = oracle_mod.sort_radix_parallel(k, v)
        r = stable_reference(k, v)
        assert np.array_equal(a[1], r[1]) and np.array_equal(b[1], r[1])


def test_radix_parallel_key_bits(oracle_mod):
    rng = np.random.default_rng(3)
    k = rng.integers(0, 1 << 20, 100_000, dtype=np.uint32)
    v = np.arange(k.size, dtype=np.uint32)
    ks, vs = oracle_mod.sort_radix_parallel(k, v, key_bits=20)
    assert np.array_equal(vs, np.argsort(k, kind="stable"))


def _rest_density_run(oracle_mod):
    p, pos = scene.rest_density_scene()
    o = oracle_mod.Oracle(p, pos)
    assert o.n == 4800 and o.T == 8192
    o.run("neighbor_search")
    o.run("density_alpha")
    return p, pos, o


def test_rest_density_multiset(oracle_mod):
    """IEEE division: the sorted multiset equals the golden vector."""
    ref = np.load(os.path.join(GOLDEN, "rest_density.npy"))
    _, _, o = _rest_density_run(oracle_mod)
    rho = o.field(_abi.FE_FIELD_DENSITY)
    rel = np.abs(np.sort(rho) - np.sort(ref)) / np.sort(ref)
    assert rel.max() < 2e-6
    # published summary (implementation.tex / plot_rest_density.py)
    assert abs(rho.min() - 606.560181) < 1e-3
    assert abs(rho.max() - 999.974548) < 2e-3
    assert abs(float(rho.mean()) - 945.91) < 0.01


def test_rest_density_elementwise_with_driver_division(oracle_mod):
    """The Vulkan driver computed floor(p / h) as floor(p * (1/h)); with that
    cell assignment the bitonic network reproduces the golden order exactly,
    and every density matches within FP32 summation-order noise."""
    ref = np.load(os.path.join(GOLDEN, "rest_density.npy"))
    p, pos, o = _rest_density_run(oracle_mod)
    rho = o.field(_abi.FE_FIELD_DENSITY)
    idx = o.field(_abi.FE_FIELD_ENTRY_INDEX)[:4800]
    by_particle = np.empty(4800, np.float32)
    by_particle[idx] = rho
    h = np.float32(p.smoothing_radius)
    cells = np.floor(pos * (np.float32(1.0) / h)).astype(np.int64).astype(np.uint32)
    with np.errstate(over="ignore"):
        key = ((cells[:, 0] * np.uint32(73856093)) ^ (cells[:, 1] * np.uint32(19349663))
               ^ (cells[:, 2] * np.uint32(83492791))) % np.uint32(8192)
    k, v = padded(key)
    _, vs = oracle_mod.sort_bitonic(k, v)
    guess = by_particle[vs[:4800]]
    rel = np.abs(guess - ref) / ref
    assert rel.max() < 2e-6, rel.max()


def test_det_sum_order_and_value(oracle_mod):
    rng = np.random.default_rng(11)
    for n in (1, 255, 256, 257, 70_000, 300_001):
        x = rng.random(n) * 1000
        s = oracle_mod.det_sum(x)
        assert abs(s - math.fsum(x)) <= 1e-12 * abs(math.fsum(x)) * 10
        # a pure-Python restatement of the order
        a = np.zeros(((n + 255) // 256) * 256)
        a[:n] = x

        def tree(v):
            v = v.copy()
            w = []
            for wi in range(8):
                s_ = v[32 * wi:32 * wi + 32].copy()
                m = 16
                while m:
                    s_[:m] = s_[:m] + s_[m:2 * m]
                    m //= 2
                w.append(s_[0])
            w = np.array(w)
            m = 4
            while m:
                w[:m] = w[:m] + w[m:2 * m]
                m //= 2
            return w[0]

        parts = np.array([tree(a[c * 256:(c + 1) * 256]) for c in range(len(a) // 256)])
        fin = np.zeros(256)
        for t in range(256):
            acc = 0.0
            for c in range(t, len(parts), 256):
                acc = acc + parts[c]
            fin[t] = acc
        assert tree(fin) == s


def test_oracle_thread_invariance(oracle_mod):
    w = scene.workload("dam_break_16k")
    pos = w.positions()
    outs = []
    for t in (1, 4):
        oracle_mod.set_threads(t)
        o = oracle_mod.Oracle(w.params, pos)
        o.step(2)
        outs.append((o.field(_abi.FE_FIELD_POSITION_A), o.field(_abi.FE_FIELD_PRESSURE),
                     o.field(_abi.FE_FIELD_VELOCITY_A)))
    oracle_mod.set_threads(0)
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_fp32_against_fp64_twin(oracle_mod):
    """The FP32 restatement stays close to the FP64 twin over one step."""
    w = scene.workload("dam_break_16k")
    pos = w.positions()
    a = oracle_mod.Oracle(w.params, pos)
    b = oracle_mod.Oracle(w.params, pos, fp64=True)
    a.step(1)
    b.step(1)
    # same sort permutation at this horizon
    assert np.array_equal(a.field(_abi.FE_FIELD_ENTRY_INDEX), b.field(_abi.FE_FIELD_ENTRY_INDEX))
    rho32 = a.field(_abi.FE_FIELD_DENSITY).astype(np.float64)
    rho64 = b.field(_abi.FE_FIELD_DENSITY, f64=True)
    assert np.max(np.abs(rho32 - rho64) / rho64) < 1e-5
    p32 = a.field(_abi.FE_FIELD_POSITION_A)[:, :3].astype(np.float64)
    p64 = b.field(_abi.FE_FIELD_POSITION_A, f64=True).reshape(-1, 4)[:, :3]
    assert np.max(np.abs(p32 - p64)) < 1e-5


def test_reference_mode_divergence_quirk(oracle_mod):
    """Q2: in REFERENCE mode the divergence correction lands in velocity_a
    (previous order) and the next viscosity reads velocity_b, so the
    divergence solve cannot change positions; FIXED mode makes it count."""
    w = scene.workload("dam_break_16k")
    pos = w.positions()
    res = {}
    for mode in (_abi.FE_MODE_REFERENCE, _abi.FE_MODE_FIXED):
        for kd in (0, 4):
            p = _abi.copy_params(w.params)
            p.mode = mode
            p.divergence_solver_iterations = kd
            o = oracle_mod.Oracle(p, pos)
            o.step(3)
            res[(mode, kd)] = o.field(_abi.FE_FIELD_POSITION_A)
    assert np.array_equal(res[(0, 0)], res[(0, 4)])
    assert not np.array_equal(res[(1, 0)], res[(1, 4)])


def test_stats_fixed_point(oracle_mod):
    w = scene.workload("dam_break_16k")
    o = oracle_mod.Oracle(w.params, w.positions())
    st = o.step(2)
    rho = o.field(_abi.FE_FIELD_DENSITY)
    src = o.field(_abi.FE_FIELD_SOURCE_TERM)
    vel = o.field(_abi.FE_FIELD_VELOCITY_A)
    de = np.abs(rho - np.float32(1000.0))
    expect1 = int(np.minimum(np.floor(de).astype(np.int64), 10000).sum()) & 0xFFFFFFFF
    expect2 = int(np.minimum(np.floor(np.abs(src) * np.float32(10.0)).astype(np.int64),
                             10000).sum()) & 0xFFFFFFFF
    assert st.density_error_fp == expect1 and st.divergence_error_fp == expect2
    sp = np.sqrt((vel[:, 0] * vel[:, 0] + vel[:, 1] * vel[:, 1]) + vel[:, 2] * vel[:, 2])
    assert st.max_speed == np.float32(sp.max())
    assert abs(st.avg_density_error_f64 - np.mean(np.abs(rho.astype(np.float64) - 1000.0))) < 1e-9


def test_oracle_splat_weights_and_clipping(oracle_mod):
    """One particle in the middle of a 32^3 grid receives the full 17^3 stencil:
    the sum equals the sum of the shader's weights over offsets with d < 8; a
    particle beyond box_max adds nothing."""
    import numpy as np

    from fluid_step import _abi
    p = _abi.default_params()
    p.box_min[:] = [0.0, 0.0, 0.0]
    p.box_max[:] = [1.0, 1.0, 1.0]
    p.grid_res[:] = [32, 32, 32]
    pos = np.array([[0.5, 0.5, 0.5, 1.0], [1.5, 0.5, 0.5, 1.0]], np.float32)
    g = oracle_mod.splat_density(pos, p)
    total = 0
    for z in range(-8, 9):
        for y in range(-8, 9):
            for x in range(-8, 9):
                d = np.float32(np.sqrt(np.float32(np.float32(x * x + y * y) + z * z)))
                if d < 8:
                    xn = np.float32(d / np.float32(8))
                    wt = np.float32(1) - xn * xn
                    wt = np.float32(np.float32(wt * wt) * wt)
                    total += int(np.float32(wt * np.float32(200)))
    assert int(g.sum()) == total
    assert g[16, 16, 16] == 200 and g[16, 16, 24] == 0
