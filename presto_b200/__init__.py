"""presto_b200: B200-native Fourier-domain acceleration/jerk search engine,
a drop-in for the hot path of PRESTO's accelsearch.

The compute lives in libaccel_b200.so (CUDA for sm_100a + host C) behind the
C ABI in include/accel_b200.h; this package is its Python host mirror.
"""
from .accel import (CORR_FFT, CORR_TC_SPLIT_BF16, CORR_TC_SPLIT_FP16, AccelError, AccelSearch, CandList,  # noqa: F401
                    Context, algorithmic_counts,
                    bank_geometry, candidate_sigma, eliminate_harmonics, lib, make_params,
                    get_fourier_amplitudes, get_transform_costs, num_blocks, obs_init,
                    power_for_sigma, FourierProps, RzwErrs, calc_props, calc_rzwerrs, cand_props,
                    read_candfile, write_candfile, write_accelfile, accel_filenames, nice_output,
                    set_transform_costs, sort_cands, read_zaplist, zapbirds_host, mt19937_output,
                    dedisp_delays)
