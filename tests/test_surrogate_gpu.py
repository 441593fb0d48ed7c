"""Surrogate on the GPU: the tcgen05 bf16 GEMM against a PyTorch fp32 matmul
of the same bf16 operands, features / forward / gradients / Adam against the
NumPy oracle, and online training that learns to rank real decodes."""
import ctypes

import numpy as np
import pytest

from brkga_fft2_b200 import abi, instances, pack_problem
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required")
    from brkga_fft2_b200 import build
    build.build()
    return torch


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (256, 512, 320), (512, 320, 256), (384, 256, 512)])
def test_gemm_bf16_matches_fp32_matmul(torch, M, N, K):
    lib = abi.load_library()
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C = torch.full((M, N), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = lib.brkga_gemm_bf16(ctypes.c_void_p(A.data_ptr()), K, ctypes.c_void_p(B.data_ptr()), K,
                             ctypes.c_void_p(C.data_ptr()), N, M, N, K, ctypes.c_void_p(err.data_ptr()),
                             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = A.float() @ B.float().T  # fp32 reference of the same bf16 operands
    torch.testing.assert_close(C, ref, rtol=1e-4, atol=1e-3)


@pytest.fixture(scope="module")
def p100(torch):
    from brkga_fft2_b200.evaluator import DeviceDecoder
    from brkga_fft2_b200.surrogate import Surrogate
    inst = instances.p100m4(0)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    dd = DeviceDecoder(pk, max_pop=4096)
    sur = Surrogate(dd.native, max_batch=1024, buffer_capacity=20000, seed=7)
    return inst, pk, dd, sur


def test_features_match_oracle(torch, p100):
    inst, pk, dd, sur = p100
    ch = instances.chromosomes(40, inst.nb_parts, 3)
    got = sur.features(torch.from_numpy(ch).cuda())
    ref = mo.features(pk, ch, sur.in_pad)
    assert sur.in_features == 3 * inst.nb_parts + 2 * inst.nb_machines
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("workload", ["p50m2", "p200m6", "p400m8"])
def test_features_match_oracle_across_sizes(torch, workload):
    """Both feature kernels (one warp per chromosome up to 256 parts, one CTA
    per chromosome beyond) against the oracle, with tied sequencing keys, a
    NaN machine key (the part matches no machine) and keys on the float32
    thresholds."""
    from brkga_fft2_b200.evaluator import DeviceDecoder
    from brkga_fft2_b200.surrogate import Surrogate
    inst = getattr(instances, workload)(0)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    dd = DeviceDecoder(pk, max_pop=64)
    N = inst.nb_parts
    ch = instances.chromosomes(37, N, 21)
    ch[0, :7] = ch[0, 7]
    ch[1, N + 3] = np.float32(np.nan)
    ch[2, N:N + 4] = np.float32(1.0 / inst.nb_machines)
    for kind, ref in (("decode", mo.features), ("order", mo.order_features)):
        sur = Surrogate(dd.native, max_batch=128, buffer_capacity=1000, seed=3, features=kind)
        got = sur.features(torch.from_numpy(ch).cuda())
        np.testing.assert_array_equal(got, ref(pk, ch, sur.in_pad))
        sur.close()


def test_order_features_match_oracle(torch, p100):
    """The screened configuration's input (per part its sequencing key, area
    and height, parts sorted by key); here P100M4: 300 values."""
    from brkga_fft2_b200.surrogate import Surrogate
    inst, pk, dd, _ = p100
    sur = Surrogate(dd.native, max_batch=256, buffer_capacity=1000, seed=3, features="order")
    assert sur.in_features == 3 * inst.nb_parts and sur.in_pad == 320
    ch = instances.chromosomes(40, inst.nb_parts, 5)
    ch[0, :10] = ch[0, 10]  # tied keys keep gene order
    got = sur.features(torch.from_numpy(ch).cuda())
    np.testing.assert_array_equal(got, mo.order_features(pk, ch, sur.in_pad))
    sur.close()


def test_forward_gradients_adam_match_oracle(torch, p100):
    from brkga_fft2_b200.surrogate import split_params
    inst, pk, dd, sur = p100
    B, n = 256, 201
    ch = instances.chromosomes(B, inst.nb_parts, 4)
    X = mo.features(pk, ch, sur.in_pad)
    t = np.random.default_rng(0).normal(size=B).astype(np.float32)
    Xb = torch.from_numpy(X.astype(np.float32)).cuda().to(torch.bfloat16)
    sur.load_batch(Xb, torch.from_numpy(t).cuda(), n)
    sur.gradients(B)
    flat = sur.params().astype(np.float64)
    p = split_params(flat, sur.in_pad)
    y_ref, _ = mo.forward(p, X, bf=True)
    np.testing.assert_allclose(sur.predictions(B), y_ref, rtol=2e-3, atol=2e-3)
    g = split_params(sur.grads().astype(np.float64), sur.in_pad)
    gr = mo.grads(p, X, t.astype(np.float64), n, bf=True)
    for name in gr:
        rel = np.linalg.norm(g[name] - gr[name]) / max(np.linalg.norm(gr[name]), 1e-12)
        assert rel < 2e-2, (name, rel)
    # one Adam step from zero moments
    sur.adam(1e-3)
    new = sur.params().astype(np.float64)
    w, _, _ = mo.adam(flat, sur.grads().astype(np.float64), 0.0, 0.0, 1, 1e-3)
    np.testing.assert_allclose(new, w, rtol=1e-5, atol=1e-6)


def test_online_training_learns_to_rank(torch, p100):
    from brkga_fft2_b200.surrogate import spearman
    inst, pk, dd, sur = p100
    train = torch.from_numpy(instances.chromosomes(4096, inst.nb_parts, 10)).cuda()
    ms = dd.decode(train)
    sur.observe(train, ms)
    test = torch.from_numpy(instances.chromosomes(1000, inst.nb_parts, 11)).cuda()
    exact = dd.decode(test).cpu().numpy()
    before = spearman(sur.predict(test).cpu().numpy(), exact)
    sur.train(300, batch=512, lr=1e-3)
    after = spearman(sur.predict(test).cpu().numpy(), exact)
    assert after > 0.7 and after > before + 0.2, (before, after)


def test_observe_fills_ring_in_row_order(torch, p100):
    """Feasible rows (finite, below 1e15) take ring slots in row order, across
    the 1024-row passes of one call and across calls, wrapping at capacity;
    infeasible and NaN rows take none."""
    from brkga_fft2_b200.surrogate import Surrogate
    inst, pk, dd, _ = p100
    cap = 3000
    sur = Surrogate(dd.native, max_batch=1024, buffer_capacity=cap, seed=1)
    rng = np.random.default_rng(5)
    ms = rng.uniform(5e5, 9e5, 5000)
    ms[::7] = 1e16
    ms[3::11] = np.nan
    ch = torch.from_numpy(instances.chromosomes(5000, inst.nb_parts, 4)).cuda()
    msd = torch.from_numpy(ms).cuda()
    sur.observe(ch[:2500], msd[:2500])
    sur.observe(ch[2500:], msd[2500:])
    torch.cuda.synchronize()
    norm = sur._io(5, np.zeros(3, np.float64), False)
    count = sur._io(9, np.zeros(1, np.int64), False)
    ring = sur._io(8, np.zeros(cap, np.float32), False)
    feas = np.isfinite(ms) & (ms < 1e15)
    first = ms[:2500][feas[:2500]]
    assert norm[2] == 1.0
    assert norm[0] == pytest.approx(first.mean(), rel=1e-12)
    assert int(count[0]) == int(feas.sum())
    want = np.full(cap, np.nan, np.float32)
    for k, v in enumerate(ms[feas]):
        want[k % cap] = np.float32((v - norm[0]) / norm[1])
    np.testing.assert_array_equal(ring, want)


def test_gemm_bf16_refuses_misaligned_operands(torch):
    """The operands are loaded by TMA: a base address that is not 16-byte
    aligned is refused before anything is launched."""
    lib = abi.load_library()
    A = torch.zeros(128 * 64 + 8, dtype=torch.bfloat16, device="cuda")
    B = torch.zeros(64, 64, dtype=torch.bfloat16, device="cuda")
    C = torch.zeros(128, 64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    bad = ctypes.c_void_p(A.data_ptr() + 2)  # one bf16 element off a 16-byte boundary
    st = lib.brkga_gemm_bf16(bad, 64, ctypes.c_void_p(B.data_ptr()), 64, ctypes.c_void_p(C.data_ptr()), 64,
                             128, 64, 64, ctypes.c_void_p(err.data_ptr()), s)
    assert st == abi.ERR_INVALID_ARGUMENT
    st = lib.brkga_gemm_bf16(ctypes.c_void_p(A.data_ptr()), 64, ctypes.c_void_p(B.data_ptr()), 64,
                             ctypes.c_void_p(C.data_ptr()), 64, 128, 64, 64, ctypes.c_void_p(err.data_ptr()), s)
    assert st == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
