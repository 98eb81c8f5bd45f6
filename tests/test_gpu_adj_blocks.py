"""GPU parity of the discrete adjoint's building blocks: J v, J^T v
(Jac_SP_Vec / JacTR_SP_Vec) and the transposed LU solve (KppSolveTR), as
kpp_b200_jac_vec / kpp_b200_solve_tr compute them for a batch, against the
reference's generated C functions cell by cell.  No libm function is
involved, so the bar is bit-identity."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


@pytest.mark.parametrize("mech", ["small_strato", "saprc99", "mcm_isoprene"])
def test_jacobian_products_and_transposed_solve_bit_identical(mech, golden_dir):
    from kpp_b200 import build, load
    from oracle_lib import OracleLib, lib_path
    if mech in build.ON_REQUEST and not build.library_path(mech).exists():
        pytest.skip(f"{mech} is built on request")
    if not lib_path(mech).exists():
        pytest.skip("oracle libraries not present")
    m = load(mech)
    o = OracleLib(mech)
    ref = o.lib
    for nm in ("Jac_SP_Vec", "JacTR_SP_Vec", "KppSolveTR"):
        getattr(ref, nm).argtypes = [ctypes.c_void_p] * 3
    ref.KppDecomp.argtypes = [ctypes.c_void_p]
    diag = o.lu_pattern()[3][: o.nvar]
    g = np.load(golden_dir / f"funjac_{mech}.npz")
    jvs = np.ascontiguousarray(g["jvs"])  # [LU_NONZERO, n]
    n = jvs.shape[1]
    rng = np.random.default_rng(12)
    uv = rng.standard_normal((o.nvar, n))
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    for transposed, ref_fn in ((False, ref.Jac_SP_Vec), (True, ref.JacTR_SP_Vec)):
        got = m.jac_vec(d(jvs), d(uv), transposed=transposed).cpu().numpy()
        for c in range(n):
            # named arrays: the pointers handed to C must outlive the call
            jc, uc = np.ascontiguousarray(jvs[:, c]), np.ascontiguousarray(uv[:, c])
            want = np.zeros(o.nvar)
            ref_fn(_p(jc), _p(uc), _p(want))
            np.testing.assert_array_equal(got[:, c], want)
    # factorised Rosenbrock matrices 1/(h gamma) - J, factorised by the reference
    e = -jvs.copy()
    e[diag, :] += 1.0 / (10.0 * 0.5)
    ok = []
    for c in range(n):
        col = np.ascontiguousarray(e[:, c])
        ok.append(ref.KppDecomp(_p(col)) == 0)
        e[:, c] = col
    x = rng.standard_normal((o.nvar, n))
    got = m.solve_tr(d(e), d(x)).cpu().numpy()
    assert any(ok)
    for c in range(n):
        if not ok[c]:
            continue
        ec, xc = np.ascontiguousarray(e[:, c]), np.ascontiguousarray(x[:, c])
        want = np.zeros(o.nvar)
        ref.KppSolveTR(_p(ec), _p(xc), _p(want))
        np.testing.assert_array_equal(got[:, c], want)
    # in place, as the reference's adjoint integrators call it
    # (KppSolveTR(A, b, b)): the output aliases the right-hand side
    xd = d(x)
    got_in_place = m.solve_tr(d(e), xd, out=xd).cpu().numpy()
    for c in range(n):
        if not ok[c]:
            continue
        ec = np.ascontiguousarray(e[:, c])
        xc = np.ascontiguousarray(x[:, c])
        ref.KppSolveTR(_p(ec), _p(xc), _p(xc))
        np.testing.assert_array_equal(got_in_place[:, c], xc)
