"""B200-native (sm_100a) DQMC sweep for sun-hubbard (YuanyueChen/sunhubbardmy).

The hot path -- local HS updates, time-slice wrap, UDV-stabilised Green's
function and equal-time measurement of the finite-temperature sweep, and the
projective (ground-state) sweep with the t-V bond field -- runs in
``_lib/libdqmc_gpu.so`` behind the C ABI of ``include/dqmc_gpu.h``.  This
package is the Python host mirror of the reference's driver and operator
procedures; there is no CPU fallback: every call goes through the CUDA
library and fails loudly if it is missing.
"""
from .dqmc import (  # noqa: F401
    CHAIN, CHECKERBOARD, CUBIC, R_CUBIC, DELAY, DENSE, FAST, FFT, GENERAL4, EXACT, HONEYCOMB, SQUARE, SUBMATRIX,
    EINVAL, ECUDA, ENOMEM, ESTATE, ENUMERIC, EWRAP, FAIL_NONFINITE, FAIL_SINGULAR, FAIL_WRAP,
    Dqmc, DqmcError, DqmcParams, lib_path, load_library, qr_logdet_noalloc, read_dqmc_in, sweep_start_concurrent, sweeps_concurrent,
    test_seed, trial_state,
)
from .io import (  # noqa: F401
    dyn_output, dyn_output3d, equaltime_output, equaltime_output3d, read_conf, unpack_bins, write_conf,
)
