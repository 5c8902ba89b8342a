"""Comparison helpers shared by the parity tests (vectorised, so they run on the 4.2M-row model)."""
import numpy as np


def rel_err(a, ref):
    """max |a - ref| / max |ref|."""
    return float(np.abs(np.asarray(a) - np.asarray(ref)).max() / np.abs(ref).max())


def row_scale(A):
    """Largest |entry| of each row of a system in the split layout (D, AU/INU, AL/INL)."""
    n = A.D.shape[0]
    scale = np.abs(A.D).copy()
    ru = np.repeat(np.arange(n), np.diff(A.INU))
    rl = np.repeat(np.arange(n), np.diff(A.INL))
    np.maximum.at(scale, ru, np.abs(A.AU))
    np.maximum.at(scale, rl, np.abs(A.AL))
    return scale, ru, rl


def assert_system_close(sys_gpu, A, rtol=1e-12):
    """Entries within rtol of the row's largest entry, the curl-curl (real) part bit-exact."""
    scale, ru, rl = row_scale(A)
    assert np.all(np.abs(sys_gpu["D"] - A.D) <= rtol * scale)
    assert np.all(np.abs(sys_gpu["AU"] - A.AU) <= rtol * scale[ru])
    assert np.all(np.abs(sys_gpu["AL"] - A.AL) <= rtol * scale[rl])
    # the real part (curl-curl) is computed in the reference's operation order: bit-exact
    assert np.array_equal(sys_gpu["D"].real, A.D.real)
    assert np.array_equal(sys_gpu["AU"].real, A.AU.real)
    bscale = np.abs(A.b).max()
    assert np.all(np.abs(sys_gpu["b"] - A.b) <= rtol * bscale)
