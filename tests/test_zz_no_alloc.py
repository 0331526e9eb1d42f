"""The allocation-free QR entry point (dqmc_gpu_qr_logdet_noalloc).

It exists for host codes that cannot allocate device memory themselves: their
device memory comes from a pool they do not control, or they must not
allocate once a run has started.  The entry point uses only the caller's
buffers and a fixed scratch area compiled into the library.  This test gives
it caller-owned device buffers (allocated here by torch, standing in for such
a caller's pool), calls it twice in a row through the C ABI, and checks each
result against the handle-based QR entry point (dqmc_gpu_test_qr) on the same
matrix.  Tolerance: 1e-12 relative, as for the other tensor-core parity tests.

The file name makes pytest collect it after every other test module.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _graded(n, seed):
    rng = np.random.default_rng(seed)
    a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) * np.logspace(6, -6, n)[None, :]
    return np.asfortranarray(a)


def _reference_qr(sb, a):
    """QR through the existing handle-based entry point (a handle whose chain
    has N = n sites: a square lattice when n is a square, else a honeycomb one)."""
    n = a.shape[0]
    side = int(round(np.sqrt(n)))
    if side * side == n:
        p = sb.DqmcParams.make(lattice=1, l1=side, l2=side, beta=1.0, dtau=0.1, rhub=4.0, nwrap=10)
    else:
        side = int(round(np.sqrt(n // 2)))
        assert 2 * side * side == n
        p = sb.DqmcParams.make(lattice=2, l1=side, l2=side, beta=1.0, dtau=0.1, rhub=4.0, nwrap=10)
    with sb.Dqmc(p, 1) as g:
        g.set_work(0, a)
        ld = g.test_qr(0, 1)[0]
        return g.work(0), g.work(1), ld


def _rel(x, y):
    return float(np.max(np.abs(x - y)) / max(1e-300, np.max(np.abs(y))))


# 64 and 256 fill whole 16-column panels and 64-column blocks; 36, 100 and
# 484 end on a ragged panel (n mod 16 = 4); 512 is the scratch limit
@pytest.mark.parametrize("n", [36, 64, 100, 256, 484, 512])
def test_noalloc_qr_matches_handle_qr_twice(n):
    import torch
    import sunhubbardmy_b200 as sb

    torch.cuda.set_device(0)
    mats = [_graded(n, 11), _graded(n, 12)]
    # caller-owned device buffers, column-major complex128 (transpose trick:
    # a C-contiguous torch tensor of shape (n, n) holding A^T is A in Fortran order)
    a_dev = torch.empty((n, n), dtype=torch.complex128, device="cuda")
    q_dev = torch.empty((n, n), dtype=torch.complex128, device="cuda")
    ld_dev = torch.empty(1, dtype=torch.complex128, device="cuda")
    for a in mats:                      # two calls in a row on the same scratch
        a_dev.copy_(torch.from_numpy(np.ascontiguousarray(a.T)))
        sb.qr_logdet_noalloc(n, a_dev.data_ptr(), q_dev.data_ptr(), ld_dev.data_ptr(), 0)
        torch.cuda.synchronize()
        f_new = a_dev.cpu().numpy().T
        q_new = q_dev.cpu().numpy().T
        ld_new = complex(ld_dev.cpu().numpy()[0])
        f_ref, q_ref, ld_ref = _reference_qr(sb, a)
        assert _rel(np.triu(f_new), np.triu(f_ref)) < TOL
        assert _rel(q_new, q_ref) < TOL
        assert abs(ld_new - ld_ref) < 1e-10
        # and it is a QR factorisation of a
        r = np.triu(f_new)
        col = np.max(np.abs(a), axis=0)
        assert np.max(np.abs(q_new @ r - a) / col[None, :]) < 1e-12


def test_noalloc_rejects_oversize():
    import sunhubbardmy_b200 as sb
    with pytest.raises(sb.DqmcError, match="outside 1..512"):
        sb.qr_logdet_noalloc(513, 1, 1, 1, 0)
