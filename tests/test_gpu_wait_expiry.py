"""The expiry path of the tensor-core kernels' bounded waits, on the GPU.

Every mbarrier wait of the INT8 FP64-accurate matvec (oz_mma_kernel), the
3xTF32 matvec (pk_tc_kernel) and the tensor-core Gram of the factor
(gram_tc_kernel) is a bounded poll.  mbc_solver_set_wait_limit shortens the
waits for a partner role or a copy to one poll, so that they expire on a
normal launch.  The kernel must then stop, wait with the default limit for
its own bulk copies and MMAs, free its tensor memory and return; the call
reports MBC_TIMEOUT.  With the default limit restored, the same call on the
same solver must give the same result as before the failure, bit for bit
(the kernels are deterministic): a CTA that had left tensor memory
allocated, or a copy still landing, would instead stall or corrupt the next
launch.  Nothing here faults, traps or hangs a GPU: the waits stay bounded,
only their bound is small.
"""
import numpy as np
import pytest

import fastmbcui_b200 as F
from fastmbcui_b200 import scenes as S
from fastmbcui_b200._lib import MBC_TIMEOUT

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _d(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")


def _expect_timeout(call, tries=3):
    """`call` under a one-poll limit reports MBC_TIMEOUT (a launch whose waits
    all happened to find their phase complete on the first poll is retried)."""
    for _ in range(tries):
        try:
            call()
        except F.MbcError as e:
            assert e.status == MBC_TIMEOUT, e
            return
    pytest.fail("no bounded wait expired under a one-poll limit")


@pytest.fixture(scope="module")
def scene():
    sc = S.ellipsoids_scene(3, 2000, seed=9)
    return sc, F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)


def test_int8_matvec_wait_expiry(scene):
    sc, plan = scene
    s = F.Solver(plan, x=_d(sc.x), nx=_d(sc.nx), y=_d(sc.y), coef=sc.coef, precision=F.MBC_F64)
    s.set_fp64_matvec("int8").prepare()  # digit planes and the first-use check, at the default limit
    V = _d(np.random.default_rng(0).standard_normal((sc.n, 48)), torch.float64)
    ref_k, ref_kt = s.apply_K(V), s.apply_KT(_d(np.ones((sc.nf, 48)), torch.float64))
    s.set_wait_limit(1)
    _expect_timeout(lambda: s.apply_K(V))
    _expect_timeout(lambda: s.apply_KT(_d(np.ones((sc.nf, 48)), torch.float64)))
    s.set_wait_limit(0)
    assert torch.equal(s.apply_K(V), ref_k)
    assert torch.equal(s.apply_KT(_d(np.ones((sc.nf, 48)), torch.float64)), ref_kt)


def test_tf32_matvec_wait_expiry(scene):
    sc, plan = scene
    s = F.Solver(plan, x=_d(sc.x), nx=_d(sc.nx), y=_d(sc.y), coef=sc.coef, precision=F.MBC_F32)
    s.set_matvec(F.MBC_MATVEC_TENSOR)
    V = _d(np.random.default_rng(1).standard_normal((sc.n, 32)))
    ref = s.apply_K(V)
    s.set_wait_limit(1)
    _expect_timeout(lambda: s.apply_K(V))
    s.set_wait_limit(0)
    assert torch.equal(s.apply_K(V), ref)


def test_tensor_gram_wait_expiry(scene):
    sc, plan = scene
    s = F.Solver(plan, x=_d(sc.x), nx=_d(sc.nx), y=_d(sc.y), coef=sc.coef, precision=F.MBC_F32)
    s.set_factor_tiles(dict(s.factor_tiles(), tc_min_ns=32))
    ref, _ = s.factor().get_factor()
    assert s.tensor_grams() > 0
    s.set_wait_limit(1)
    _expect_timeout(lambda: s.factor())
    s.set_wait_limit(0)
    got, _ = s.factor().get_factor()
    assert np.array_equal(got, ref)
