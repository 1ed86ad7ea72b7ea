"""Python host mirror of the accelsearch hot path over the C ABI of
libaccel_b200.so (include/accel_b200.h).

Names, argument meanings and defaults follow PRESTO's accelsearch
(clig/accelsearch_cmd.cli, src/accel_utils.c).  Every compute call goes to
the CUDA engine; there is no CPU fallback: a missing library or a missing
GPU raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libaccel_b200.so")

AB_OK = 0
ERRORS = {-1: "AB_ERR_ARG", -2: "AB_ERR_CUDA", -3: "AB_ERR_NOMEM", -4: "AB_ERR_OVERFLOW",
          -5: "AB_ERR_STATE", -6: "AB_ERR_BUDGET"}

# Every symbol include/accel_b200.h declares.
EXPORTS = [
    "ab_params_default", "ab_ctx_create", "ab_ctx_destroy", "ab_ctx_last_error",
    "ab_ctx_stream", "ab_ctx_set_hbm_budget", "ab_obs_init", "ab_prepare", "ab_search",
    "ab_last_hits", "ab_last_cands", "ab_set_spectrum", "ab_subharm_fderivs_vol", "ab_add_ffdotpows",
    "ab_fund_to_ffdotplane", "ab_inmem_add_ffdotpows", "ab_candlist_new", "ab_candlist_free",
    "ab_candlist_get", "ab_candlist_insert", "ab_search_ffdotpows", "ab_block_stage_sums", "ab_gen_response",
    "ab_bank_kernel", "ab_candidate_sigma", "ab_power_for_sigma", "ab_chi2_logp",
    "ab_equivalent_gaussian_sigma", "ab_sort_cands", "ab_eliminate_harmonics",
    "ab_ctx_set_profiling", "ab_ctx_kernel_times", "ab_ctx_reset_kernel_times",
    "ab_ctx_launch_count", "ab_bank_geometry", "ab_num_blocks_main", "ab_measure_fp32_peak",
    "ab_fderivs_vol_noalloc", "ab_pool_create", "ab_pool_destroy", "ab_pool_last_error",
    "ab_pool_submit", "ab_pool_wait", "ab_pool_stats", "ab_pool_reset_stats", "ab_tc_gemm",
    "ab_ctx_set_corr_path", "ab_w_resp_halfwidth", "ab_set_transform_costs",
    "ab_get_transform_costs", "ab_autotune", "ab_add_ffdotpows_ptrs",
    "ab_fund_to_ffdotplane_trans", "ab_inmem_add_ffdotpows_trans", "ab_copy_ffdotpows",
    "ab_get_fourier_amplitudes", "ab_optimize_cands", "ab_realfft", "ab_deredden",
    "ab_series_to_fft", "ab_calc_props", "ab_calc_rzwerrs", "ab_cand_props",
    "ab_write_accelfile", "ab_nice_output_1", "ab_nice_output_2", "ab_set_worklog",
    "ab_last_worklog", "ab_candlist_set_worklog", "ab_candlist_worklog", "ab_ffdot_hits",
    "ab_read_zaplist", "ab_zapbirds", "ab_zapbirds_host", "ab_mt19937_output",
    "ab_pool_set_corr_path", "ab_dedisp_delays", "ab_dedisperse", "ab_search_dedispersed",
]

COST_SLOTS = 16

# correlation paths (ab_ctx_set_corr_path)
CORR_FFT = 0
CORR_TC_SPLIT_BF16 = 1
CORR_TC_SPLIT_FP16 = 2


POLISH_MAX_HARM = 32


class RDerivs(C.Structure):
    """rderivs (include/presto.h:160-168)."""
    _fields_ = [(n, C.c_double) for n in ("pow", "phs", "dpow", "dphs", "d2pow", "d2phs",
                                         "locpow")]


class Polished(C.Structure):
    _fields_ = [("numharm", C.c_int), ("pows", C.c_double * POLISH_MAX_HARM),
                ("hirs", C.c_double * POLISH_MAX_HARM), ("hizs", C.c_double * POLISH_MAX_HARM),
                ("hiws", C.c_double * POLISH_MAX_HARM), ("derivs", RDerivs * POLISH_MAX_HARM)]


class FourierProps(C.Structure):
    """fourierprops (include/presto.h:170-188); an array of it is a .cand file."""
    _fields_ = [("r", C.c_double), ("rerr", C.c_float), ("z", C.c_double), ("zerr", C.c_float),
                ("w", C.c_double), ("werr", C.c_float)] + \
               [(n, C.c_float) for n in ("pow", "powerr", "sig", "rawpow", "phs", "phserr", "cen",
                                         "cenerr", "pur", "purerr", "locpow")]


class RzwErrs(C.Structure):
    """rzwerrs (include/presto.h:233-246)."""
    _fields_ = [(n, C.c_double) for n in ("p", "pd", "pdd", "f", "fd", "fdd")] + \
               [(n, C.c_float) for n in ("perr", "pderr", "pdderr", "ferr", "fderr", "fdderr")]


class AccelError(RuntimeError):
    pass


class Params(C.Structure):
    _fields_ = [("N", C.c_longlong), ("dt", C.c_double), ("numbins", C.c_longlong),
                ("zmax", C.c_int), ("wmax", C.c_int), ("wmaxP", C.c_int),
                ("numharm", C.c_int), ("sigma", C.c_float),
                ("flo", C.c_double), ("fhi", C.c_double), ("floP", C.c_int), ("fhiP", C.c_int),
                ("rlo", C.c_double), ("rhi", C.c_double), ("rloP", C.c_int), ("rhiP", C.c_int),
                ("lobin", C.c_longlong), ("inmemP", C.c_int), ("nph", C.c_float),
                ("locpowP", C.c_int), ("noharmpolishP", C.c_int)]


class Obs(C.Structure):
    _fields_ = [("N", C.c_longlong), ("numbins", C.c_longlong), ("lobin", C.c_longlong),
                ("highestbin", C.c_longlong),
                ("maxkernlen", C.c_int), ("corr_uselen", C.c_int), ("fftlen", C.c_int),
                ("numharmstages", C.c_int), ("numz", C.c_int), ("numw", C.c_int),
                ("numbetween", C.c_int), ("inmem", C.c_int), ("norm_type", C.c_int),
                ("rstep", C.c_int),
                ("dt", C.c_double), ("T", C.c_double), ("rlo", C.c_double), ("rhi", C.c_double),
                ("dr", C.c_double), ("zlo", C.c_double), ("zhi", C.c_double), ("dz", C.c_double),
                ("wlo", C.c_double), ("whi", C.c_double), ("dw", C.c_double),
                ("nph", C.c_float), ("sigma", C.c_float),
                ("powcut", C.c_float * 6), ("numindep", C.c_longlong * 6),
                ("noharmpolish", C.c_int)]


class Cand(C.Structure):
    _fields_ = [("power", C.c_float), ("sigma", C.c_float), ("numharm", C.c_int),
                ("r", C.c_double), ("z", C.c_double), ("w", C.c_double)]


class FFDotPows(C.Structure):
    _fields_ = [("rlo", C.c_longlong), ("zlo", C.c_int), ("wlo", C.c_int),
                ("numrs", C.c_int), ("numzs", C.c_int), ("numws", C.c_int),
                ("powers", C.POINTER(C.c_float)), ("capacity", C.c_size_t)]


_lib = None


def lib():
    """Loads libaccel_b200.so (built in-tree by presto_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise AccelError(f"{LIBPATH} is missing: run presto_b200.build.build() first")
    L = C.CDLL(LIBPATH)
    vp, ll, i, d = C.c_void_p, C.c_longlong, C.c_int, C.c_double
    L.ab_params_default.argtypes = [C.POINTER(Params)]
    L.ab_ctx_create.argtypes = [i, C.POINTER(vp)]
    L.ab_ctx_destroy.argtypes = [vp]
    L.ab_ctx_last_error.restype = C.c_char_p
    L.ab_ctx_last_error.argtypes = [vp]
    L.ab_ctx_stream.restype = vp
    L.ab_ctx_stream.argtypes = [vp]
    L.ab_ctx_set_hbm_budget.argtypes = [vp, C.c_size_t]
    L.ab_ctx_set_corr_path.argtypes = [vp, i]
    L.ab_w_resp_halfwidth.argtypes = [C.c_double, C.c_double]
    L.ab_set_transform_costs.argtypes = [C.POINTER(C.c_double), i]
    L.ab_get_transform_costs.argtypes = [C.POINTER(C.c_double), i]
    L.ab_autotune.argtypes = [vp, C.POINTER(C.c_double), i]
    L.ab_obs_init.argtypes = [C.POINTER(Params), C.POINTER(Obs)]
    L.ab_prepare.argtypes = [vp, C.POINTER(Obs)]
    L.ab_search.argtypes = [vp, C.POINTER(Obs), vp, i, ll, ll, C.POINTER(Cand), ll,
                            C.POINTER(ll)]
    L.ab_last_cands.argtypes = [vp, C.POINTER(Cand), ll, C.POINTER(ll)]
    L.ab_last_hits.argtypes = [vp, C.POINTER(ll), C.POINTER(i), C.POINTER(i), C.POINTER(i),
                               C.POINTER(i), C.POINTER(C.c_float), ll, C.POINTER(ll)]
    L.ab_set_spectrum.argtypes = [vp, C.POINTER(Obs), vp]
    L.ab_subharm_fderivs_vol.argtypes = [vp, C.POINTER(Obs), i, i, d, d, C.POINTER(FFDotPows)]
    L.ab_add_ffdotpows.argtypes = [vp, C.POINTER(Obs), C.POINTER(FFDotPows),
                                   C.POINTER(FFDotPows), i, i, d]
    L.ab_fund_to_ffdotplane.argtypes = [vp, C.POINTER(Obs), C.POINTER(FFDotPows)]
    L.ab_inmem_add_ffdotpows.argtypes = [vp, C.POINTER(Obs), C.POINTER(FFDotPows), i, i]
    L.ab_add_ffdotpows_ptrs.argtypes = L.ab_add_ffdotpows.argtypes
    L.ab_fund_to_ffdotplane_trans.argtypes = L.ab_fund_to_ffdotplane.argtypes
    L.ab_inmem_add_ffdotpows_trans.argtypes = L.ab_inmem_add_ffdotpows.argtypes
    L.ab_copy_ffdotpows.argtypes = [C.POINTER(FFDotPows), C.POINTER(FFDotPows)]
    L.ab_get_fourier_amplitudes.argtypes = [C.POINTER(Obs), vp, ll, i, vp]
    L.ab_optimize_cands.argtypes = [vp, C.POINTER(Obs), vp, i, C.POINTER(Cand), ll,
                                    C.POINTER(Polished)]
    L.ab_calc_props.argtypes = [C.POINTER(RDerivs), d, d, d, C.POINTER(FourierProps)]
    L.ab_calc_rzwerrs.argtypes = [C.POINTER(FourierProps), d, C.POINTER(RzwErrs)]
    L.ab_cand_props.argtypes = [C.POINTER(Cand), C.POINTER(Polished), ll, C.POINTER(FourierProps)]
    L.ab_set_worklog.argtypes = [vp, i]
    L.ab_last_worklog.argtypes = [vp, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
    L.ab_candlist_set_worklog.argtypes = [vp, i, d]
    L.ab_candlist_worklog.restype = ll
    L.ab_candlist_worklog.argtypes = [vp, C.c_char_p, C.c_size_t]
    L.ab_write_accelfile.argtypes = [C.c_char_p, C.POINTER(Obs), C.POINTER(Cand),
                                     C.POINTER(Polished), ll, C.c_char_p]
    L.ab_nice_output_1.argtypes = [C.c_char_p, C.c_size_t, d, d, i]
    L.ab_nice_output_2.argtypes = L.ab_nice_output_1.argtypes
    L.ab_realfft.argtypes = [vp, vp, ll, i, vp, i]
    L.ab_deredden.argtypes = [vp, vp, ll, i, i, d, d, i]
    L.ab_series_to_fft.argtypes = [vp, vp, ll, d, i, vp, i]
    L.ab_candlist_new.restype = vp
    L.ab_candlist_free.argtypes = [vp]
    L.ab_candlist_get.restype = ll
    L.ab_candlist_get.argtypes = [vp, C.POINTER(Cand), ll]
    L.ab_candlist_insert.argtypes = [vp, C.c_float, C.c_float, i, d, d, d]
    L.ab_search_ffdotpows.argtypes = [vp, C.POINTER(Obs), C.POINTER(FFDotPows), i, vp]
    L.ab_dedisp_delays.argtypes = [i, d, d, d, i, vp, i, i, vp, vp]
    L.ab_dedisperse.argtypes = [vp, vp, i, ll, i, d, d, d, i, vp, i, i, vp, i]
    L.ab_search_dedispersed.argtypes = [vp, vp, i, ll, i, d, d, d, i, vp, i, i, C.POINTER(Obs),
                                        C.POINTER(Cand), ll, C.POINTER(ll)]
    L.ab_read_zaplist.argtypes = [C.c_char_p, d, d, vp, vp, i, C.POINTER(i)]
    L.ab_zapbirds.argtypes = [vp, vp, i, ll, ll, vp, vp, i, C.POINTER(i)]
    L.ab_zapbirds_host.argtypes = [vp, ll, ll, vp, vp, i, C.POINTER(i)]
    L.ab_mt19937_output.restype = C.c_uint
    L.ab_mt19937_output.argtypes = [C.c_ulong, ll]
    L.ab_ffdot_hits.argtypes = [vp, C.POINTER(Obs), C.POINTER(FFDotPows), i, C.POINTER(Cand), ll,
                                C.POINTER(ll)]
    L.ab_block_stage_sums.argtypes = [vp, C.POINTER(Obs), vp, ll, vp, C.c_size_t]
    L.ab_gen_response.argtypes = [vp, d, i, d, d, i, vp]
    L.ab_bank_kernel.argtypes = [vp, C.POINTER(Obs), i, i, i, i, vp, i, C.POINTER(i)]
    for name in ("ab_candidate_sigma", "ab_power_for_sigma"):
        getattr(L, name).restype = d
        getattr(L, name).argtypes = [d, i, d]
    L.ab_chi2_logp.restype = d
    L.ab_chi2_logp.argtypes = [d, d]
    L.ab_equivalent_gaussian_sigma.restype = d
    L.ab_equivalent_gaussian_sigma.argtypes = [d]
    L.ab_sort_cands.argtypes = [C.POINTER(Cand), ll]
    L.ab_eliminate_harmonics.restype = ll
    L.ab_eliminate_harmonics.argtypes = [C.POINTER(Cand), ll]
    L.ab_ctx_set_profiling.argtypes = [vp, i]
    L.ab_ctx_kernel_times.argtypes = [vp, C.POINTER(d), C.POINTER(ll), i]
    L.ab_ctx_reset_kernel_times.argtypes = [vp]
    L.ab_bank_geometry.argtypes = [C.POINTER(Obs), C.POINTER(i), C.POINTER(i), i]
    L.ab_num_blocks_main.restype = ll
    L.ab_num_blocks_main.argtypes = [C.POINTER(Obs)]
    L.ab_measure_fp32_peak.argtypes = [vp, C.POINTER(d)]
    L.ab_tc_gemm.argtypes = [vp, vp, vp, vp, i, i, i]
    L.ab_pool_create.argtypes = [i, i, C.c_size_t, C.POINTER(vp)]
    L.ab_pool_destroy.argtypes = [vp]
    L.ab_pool_last_error.restype = C.c_char_p
    L.ab_pool_last_error.argtypes = [vp]
    L.ab_pool_submit.argtypes = [vp, C.POINTER(Params), vp, C.POINTER(ll)]
    L.ab_pool_wait.argtypes = [vp, ll, C.POINTER(Cand), ll, C.POINTER(ll), C.POINTER(d)]
    L.ab_pool_stats.argtypes = [vp, C.POINTER(ll), C.POINTER(d), C.POINTER(d), C.POINTER(d)]
    L.ab_pool_reset_stats.argtypes = [vp]
    L.ab_pool_set_corr_path.argtypes = [vp, i]
    L.ab_fderivs_vol_noalloc.argtypes = [C.POINTER(Obs), i, i, d, vp, vp, C.c_size_t, vp,
                                         C.c_size_t, vp, C.POINTER(FFDotPows)]
    L.ab_ctx_launch_count.restype = ll
    L.ab_ctx_launch_count.argtypes = [vp]
    _lib = L
    return L


def make_params(N, dt, numbins=None, zmax=200, wmax=None, numharm=8, sigma=2.0, flo=1.0,
                fhi=10000.0, rlo=None, rhi=None, inmem=False, photon=None, lobin=0,
                locpow=False, noharmpolish=False):
    """accelsearch options (src/accelsearch_cmd.c:22-61 defaults).  wmax=None
    means -wmax not given (an explicit -wmax 0 disables in-memory mode,
    src/accel_utils.c:1795); locpow=True is -locpow."""
    p = Params()
    lib().ab_params_default(C.byref(p))
    p.N, p.dt = int(N), float(dt)
    p.numbins = int(numbins if numbins is not None else N // 2)
    p.zmax, p.numharm, p.sigma = int(zmax), int(numharm), float(sigma)
    if wmax is not None:
        p.wmax, p.wmaxP = int(wmax), 1
    if rlo is not None:
        p.rlo, p.rloP, p.floP = float(rlo), 1, 0
    else:
        p.flo = float(flo)
    if rhi is not None:
        p.rhi, p.rhiP, p.fhiP = float(rhi), 1, 0
    else:
        p.fhi = float(fhi)
    p.inmemP = int(bool(inmem))
    p.nph = float(photon) if photon else 0.0
    p.lobin = int(lobin)
    p.locpowP = int(bool(locpow))
    p.noharmpolishP = int(bool(noharmpolish))
    return p


def obs_init(params):
    o = Obs()
    rc = lib().ab_obs_init(C.byref(params), C.byref(o))
    if rc:
        raise AccelError(f"ab_obs_init: {ERRORS.get(rc, rc)}")
    return o


def num_blocks(obs):
    """Blocks of the main search loop (src/accelsearch.c:187-224)."""
    return int(lib().ab_num_blocks_main(C.byref(obs)))


def bank_geometry(obs):
    """Per template bank: dict(numharm, harmnum, nz, nw, fftlen_ref, L, hw, numrs_max,
    sbm = blocks per device transform in the whole-spectrum search)."""
    n = C.c_int()
    rc = lib().ab_bank_geometry(C.byref(obs), C.byref(n), None, 0)
    if rc:
        raise AccelError(f"ab_bank_geometry: {ERRORS.get(rc, rc)}")
    info = (C.c_int * (9 * n.value))()
    lib().ab_bank_geometry(C.byref(obs), C.byref(n), info, n.value)
    keys = ("numharm", "harmnum", "nz", "nw", "fftlen_ref", "L", "hw", "numrs_max", "sbm")
    return [dict(zip(keys, info[9 * k:9 * k + 9])) for k in range(n.value)]


def get_fourier_amplitudes(obs, fft, lobin, numbins):
    """get_fourier_amplitudes: numbins bins from lobin, zero off the spectrum."""
    fft = np.ascontiguousarray(fft, dtype=np.complex64)
    out = np.zeros(numbins, np.complex64)
    rc = lib().ab_get_fourier_amplitudes(C.byref(obs), fft.ctypes.data, int(lobin), int(numbins),
                                         out.ctypes.data)
    if rc:
        raise AccelError(f"ab_get_fourier_amplitudes: {ERRORS.get(rc, rc)}")
    return out


def get_transform_costs():
    """Correlation cost per template and transform (ms) by log2 L (0: unknown)."""
    c = (C.c_double * COST_SLOTS)()
    lib().ab_get_transform_costs(c, COST_SLOTS)
    return list(c)


def set_transform_costs(costs):
    """Install a cost table (by log2 L); it chooses transform lengths and
    superblock heights of banks built afterwards."""
    c = (C.c_double * COST_SLOTS)(*[float(x) for x in list(costs)[:COST_SLOTS]])
    rc = lib().ab_set_transform_costs(c, COST_SLOTS)
    if rc:
        raise AccelError(f"ab_set_transform_costs: {ERRORS.get(rc, rc)}")


def calc_props(derivs, r, z, w):
    """calc_props (src/characteristics.c:195-264) of one rderivs (a RDerivs
    or a sequence of its 7 values)."""
    rd = derivs if isinstance(derivs, RDerivs) else RDerivs(*[float(v) for v in derivs])
    out = FourierProps()
    rc = lib().ab_calc_props(C.byref(rd), float(r), float(z), float(w), C.byref(out))
    if rc:
        raise AccelError(f"ab_calc_props: {ERRORS.get(rc, rc)} (power or local power ~ 0)")
    return out


def calc_rzwerrs(props, T):
    """calc_rzwerrs (src/characteristics.c:353-392): period, frequency, their
    derivatives and errors at the start of a run of T seconds."""
    out = RzwErrs()
    rc = lib().ab_calc_rzwerrs(C.byref(props), float(T), C.byref(out))
    if rc:
        raise AccelError(f"ab_calc_rzwerrs: {ERRORS.get(rc, rc)}")
    return out


def _cand_arrays(cands, polished):
    """ctypes arrays of (power, sigma, numharm, r, z, w) candidates and their
    polishing dicts (Context.optimize_cands)."""
    n = len(cands)
    if len(polished) != n:
        raise AccelError(f"{n} candidates but {len(polished)} polished records")
    arr = (Cand * max(n, 1))(*[Cand(c[0], c[1], c[2], c[3], c[4], c[5]) for c in cands])
    pol = (Polished * max(n, 1))()
    for k, p in enumerate(polished):
        h = len(p["pows"])
        if h > POLISH_MAX_HARM:
            raise AccelError(f"{h} harmonics: at most {POLISH_MAX_HARM}")
        pol[k].numharm = h
        zeros = np.zeros(h)
        pows, hirs, hizs, hiws = (p.get(key, zeros) for key in ("pows", "hirs", "hizs", "hiws"))
        for j in range(h):
            pol[k].pows[j] = float(pows[j])
            pol[k].hirs[j] = float(hirs[j])
            pol[k].hizs[j] = float(hizs[j])
            pol[k].hiws[j] = float(hiws[j])
            pol[k].derivs[j] = RDerivs(*[float(v) for v in p["derivs"][j]])
    return arr, pol


def cand_props(cands, polished):
    """The .cand file's records (src/accelsearch.c:261-272): per candidate
    (power, sigma, numharm, r, z, w) and its polishing (a dict from
    Context.optimize_cands), the fundamental's fourierprops at the search's
    r, z, w with the errors set to ACCEL_DR, ACCEL_DZ, ACCEL_DW / numharm."""
    n = len(cands)
    arr, pol = _cand_arrays(cands, polished)
    out = (FourierProps * max(n, 1))()
    rc = lib().ab_cand_props(arr, pol, n, out)
    if rc:
        raise AccelError(f"ab_cand_props: {ERRORS.get(rc, rc)}")
    return list(out[:n])


def write_candfile(path, props):
    """Writes fourierprops records as the reference's binary .cand file
    (src/accelsearch.c:282-284: the struct array, raw)."""
    arr = (FourierProps * len(props))(*props)
    with open(path, "wb") as f:
        f.write(bytes(arr))


def accel_filenames(rootname, obs):
    """The output names of src/accel_utils.c:1667-1682 (text, .cand and
    .txtcand) from the search's -zmax and -wmax as create_accelobs rounds them
    up (to multiples of 2 and 20); _JERK_ only when the search has w planes."""
    base = f"{rootname}_ACCEL_{int(round(obs.zhi))}"
    if obs.numw:
        base += f"_JERK_{int(round(obs.whi))}"
    return dict(accel=base, cand=base + ".cand", txtcand=base + ".txtcand")


def write_accelfile(path, obs, cands, polished, inf_path=None):
    """The text candidate file (output_fundamentals + output_harmonics,
    src/accel_utils.c:666-966) of sorted, polished candidates, with the .inf
    at inf_path appended."""
    n = len(cands)
    arr, pol = _cand_arrays(cands, polished)
    rc = lib().ab_write_accelfile(os.fsencode(path), C.byref(obs), arr, pol, n,
                                  os.fsencode(inf_path) if inf_path else None)
    if rc:
        raise AccelError(f"ab_write_accelfile: {ERRORS.get(rc, rc)}")


def nice_output(val, err, digits=1, length=0):
    """nice_output_1 / nice_output_2 (src/output.c:6-210): val(err) with a
    one- or two-digit error."""
    buf = C.create_string_buffer(512)
    f = lib().ab_nice_output_1 if digits == 1 else lib().ab_nice_output_2
    rc = f(buf, 512, float(val), float(err), int(length))
    if rc < 0:
        raise AccelError(f"nice_output_{digits}({val!r}, {err!r}): no format")
    return buf.value.decode()


def read_candfile(path):
    """The fourierprops records of a .cand file."""
    data = open(path, "rb").read()
    n = len(data) // C.sizeof(FourierProps)
    return list((FourierProps * n).from_buffer_copy(data[:n * C.sizeof(FourierProps)]))


def algorithmic_counts(obs):
    """Work of one search: f-fdot cells (numrs x numz x max(numw,1) per block
    per stage), correlation FLOPs at the reference FFT lengths
    (numz_h numw_h (5 L log2 L + 8 L) + 5 L log2 L per block and harmonic),
    harmonic-sum/search bytes when unfused (4 B per cell per stage read,
    4 B per subharmonic gather, 8 B read-modify-write per later stage) and
    the bytes the fused sum + search cannot avoid reading."""
    import math
    nb = num_blocks(obs)
    nws = max(obs.numw, 1)
    fund_cells = nb * obs.corr_uselen * obs.numz * nws
    cells = fund_cells * obs.numharmstages
    numharm = 1 << (obs.numharmstages - 1)
    flops = 0.0
    for b in bank_geometry(obs):
        L = b["fftlen_ref"]
        f = 5.0 * L * math.log2(L)
        flops += b["nz"] * b["nw"] * (f + 8.0 * L) + f
    flops *= nb
    sum_bytes = 4.0 * fund_cells * obs.numharmstages + 4.0 * fund_cells * (numharm - 1) + \
        8.0 * fund_cells * (obs.numharmstages - 1)
    # what the fused sum + search must read: in standard mode every block's
    # planes (all banks) once; in memory one value per harmonic per cell
    if obs.inmem:
        min_bytes = 4.0 * fund_cells * numharm
    else:
        min_bytes = 4.0 * nb * sum(b["nz"] * b["nw"] * b["numrs_max"] for b in bank_geometry(obs))
    # tensor-core path: 8 FLOPs per complex tap, numkern / 2 = 2 hw taps per
    # output cell, 3 products (hi.hi, hi.lo, lo.hi), numrs_max cells per row
    tc = 0.0
    hwf = lib().ab_w_resp_halfwidth
    for b in bank_geometry(obs):
        zmax, wmax = b["nz"] - 1, (b["nw"] - 1) * 10
        taps = sum(2 * hwf(float(-zmax + 2 * zi), float(-wmax + 20 * wi))
                   for wi in range(b["nw"]) for zi in range(b["nz"]))
        tc += 8.0 * 3.0 * taps * b["numrs_max"]
    return dict(blocks=nb, cells=cells, corr_flops=flops, harmsum_bytes=sum_bytes,
                harmsum_min_bytes=min_bytes, tc_flops=tc * nb)


class Context:
    """One CUDA context (device, stream, template-bank cache, scratch)."""

    def __init__(self, device=0):
        self.L = lib()
        self.ptr = C.c_void_p()
        rc = self.L.ab_ctx_create(int(device), C.byref(self.ptr))
        if rc:
            raise AccelError(f"ab_ctx_create(device={device}) failed: {ERRORS.get(rc, rc)}")

    def _check(self, rc, what):
        if rc:
            msg = self.L.ab_ctx_last_error(self.ptr)
            raise AccelError(f"{what}: {ERRORS.get(rc, rc)}: {msg.decode() if msg else ''}")

    def close(self):
        if self.ptr:
            self.L.ab_ctx_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return self.L.ab_ctx_stream(self.ptr)

    def prepare(self, obs):
        self._check(self.L.ab_prepare(self.ptr, C.byref(obs)), "ab_prepare")

    def search(self, obs, fft, first_block=0, max_blocks=-1, device_ptr=None):
        """All blocks and stages of the main search loop; returns the
        candidate list in the reference's order as a list of tuples
        (power, sigma, numharm, r, z, w)."""
        n = C.c_longlong()
        if device_ptr is not None:
            src, on_dev = C.c_void_p(device_ptr), 1
        else:
            fft = np.ascontiguousarray(fft, dtype=np.complex64)
            if fft.size < obs.numbins:
                raise AccelError("spectrum shorter than obs.numbins")
            src, on_dev = C.c_void_p(fft.ctypes.data), 0
        self._check(self.L.ab_search(self.ptr, C.byref(obs), src, on_dev, int(first_block),
                                     int(max_blocks), None, 0, C.byref(n)), "ab_search")
        cands = (Cand * max(n.value, 1))()
        self._check(self.L.ab_last_cands(self.ptr, cands, n.value, C.byref(n)), "ab_last_cands")
        return [(c.power, c.sigma, c.numharm, c.r, c.z, c.w) for c in cands[:n.value]]

    def set_worklog(self, on=True):
        """Record the .txtcand work-file lines of later searches
        (search_ffdotpows, src/accel_utils.c:1443-1447)."""
        self._check(self.L.ab_set_worklog(self.ptr, int(bool(on))), "ab_set_worklog")

    def last_worklog(self):
        """The .txtcand text of the last search (set_worklog on)."""
        n = C.c_size_t()
        self._check(self.L.ab_last_worklog(self.ptr, None, 0, C.byref(n)), "ab_last_worklog")
        buf = C.create_string_buffer(n.value + 1)
        self._check(self.L.ab_last_worklog(self.ptr, buf, n.value + 1, C.byref(n)),
                    "ab_last_worklog")
        return buf.raw[:n.value].decode()

    def last_hits(self):
        n = C.c_longlong()
        self.L.ab_last_hits(self.ptr, None, None, None, None, None, None, 0, C.byref(n))
        m = n.value
        blk = np.zeros(m, np.int64)
        st, wi, zi, ri = (np.zeros(m, np.int32) for _ in range(4))
        pw = np.zeros(m, np.float32)
        P = lambda a, t: a.ctypes.data_as(C.POINTER(t))
        self._check(self.L.ab_last_hits(self.ptr, P(blk, C.c_longlong), P(st, C.c_int),
                                        P(wi, C.c_int), P(zi, C.c_int), P(ri, C.c_int),
                                        P(pw, C.c_float), m, C.byref(n)), "ab_last_hits")
        return blk, st, wi, zi, ri, pw

    def block_stage_sums(self, obs, fft, block):
        nws = max(obs.numw, 1)
        out = np.zeros((obs.numharmstages, nws, obs.numz, obs.corr_uselen), np.float32)
        fft = np.ascontiguousarray(fft, dtype=np.complex64)
        self._check(self.L.ab_block_stage_sums(self.ptr, C.byref(obs), fft.ctypes.data,
                                               int(block), out.ctypes.data, out.size),
                    "ab_block_stage_sums")
        return out

    # ---- per-function drop-ins -------------------------------------------------
    def set_spectrum(self, obs, fft):
        fft = np.ascontiguousarray(fft, dtype=np.complex64)
        self._check(self.L.ab_set_spectrum(self.ptr, C.byref(obs), fft.ctypes.data),
                    "ab_set_spectrum")

    def subharm_fderivs_vol(self, obs, numharm, harmnum, fullrlo, fullrhi):
        f = FFDotPows()
        self.L.ab_subharm_fderivs_vol(self.ptr, C.byref(obs), numharm, harmnum, fullrlo,
                                      fullrhi, C.byref(f))        # sizes only
        need = f.numws * f.numzs * f.numrs
        buf = np.zeros(max(need, 1), np.float32)
        f.powers = buf.ctypes.data_as(C.POINTER(C.c_float))
        f.capacity = buf.size
        self._check(self.L.ab_subharm_fderivs_vol(self.ptr, C.byref(obs), numharm, harmnum,
                                                  fullrlo, fullrhi, C.byref(f)),
                    "ab_subharm_fderivs_vol")
        meta = dict(rlo=f.rlo, zlo=f.zlo, wlo=f.wlo, numrs=f.numrs, numzs=f.numzs,
                    numws=f.numws)
        return meta, buf[:need].reshape(f.numws, f.numzs, f.numrs).copy()

    @staticmethod
    def _ffd(meta, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float32)
        f = FFDotPows(meta["rlo"], meta["zlo"], meta["wlo"], meta["numrs"], meta["numzs"],
                      meta["numws"], arr.ctypes.data_as(C.POINTER(C.c_float)), arr.size)
        return f, arr

    def add_ffdotpows(self, obs, fund_meta, fund, sub_meta, sub, numharm, harmnum, fullrlo):
        ff, fa = self._ffd(fund_meta, fund.copy())
        sf, sa = self._ffd(sub_meta, sub)
        self._check(self.L.ab_add_ffdotpows(self.ptr, C.byref(obs), C.byref(ff), C.byref(sf),
                                            numharm, harmnum, fullrlo), "ab_add_ffdotpows")
        return fa

    def fund_to_ffdotplane(self, obs, meta, fund):
        f, a = self._ffd(meta, fund)
        self._check(self.L.ab_fund_to_ffdotplane(self.ptr, C.byref(obs), C.byref(f)),
                    "ab_fund_to_ffdotplane")

    def inmem_add_ffdotpows(self, obs, meta, fund, numharm, harmnum):
        f, a = self._ffd(meta, fund.copy())
        self._check(self.L.ab_inmem_add_ffdotpows(self.ptr, C.byref(obs), C.byref(f), numharm,
                                                  harmnum), "ab_inmem_add_ffdotpows")
        return a

    def search_ffdotpows(self, obs, meta, plane, numharm, candlist):
        f, a = self._ffd(meta, plane)
        self._check(self.L.ab_search_ffdotpows(self.ptr, C.byref(obs), C.byref(f), numharm,
                                               candlist.ptr), "ab_search_ffdotpows")

    def gen_response(self, kind, numbetween, numkern, z=0.0, w=0.0, roffset=0.0):
        out = np.zeros(numkern, np.complex64)
        if kind == "r":
            z, w = 0.0, 0.0
        elif kind == "z":
            w = 0.0
        self._check(self.L.ab_gen_response(self.ptr, roffset, numbetween, z, w, numkern,
                                           out.ctypes.data), "ab_gen_response")
        return out

    def bank_kernel(self, obs, numharm, harmnum, wi, zi):
        L = C.c_int()
        self._check(self.L.ab_bank_kernel(self.ptr, C.byref(obs), numharm, harmnum, wi, zi,
                                          None, 0, C.byref(L)), "ab_bank_kernel")
        out = np.zeros(L.value, np.complex64)
        self._check(self.L.ab_bank_kernel(self.ptr, C.byref(obs), numharm, harmnum, wi, zi,
                                          out.ctypes.data, L.value, C.byref(L)), "ab_bank_kernel")
        return out

    def optimize_cands(self, obs, fft, cands, device_ptr=None):
        """optimize_accelcand for (power, sigma, numharm, r, z, w) candidates of
        an acceleration search (max_rz_arr_harmonics) or, when obs.numw > 0, a
        jerk search (max_rzw_arr_harmonics): per candidate a dict of the
        harmonics' optimised pows, hirs, hizs, hiws and derivs (numharm x 7)."""
        n = len(cands)
        if n == 0:
            return []
        arr = (Cand * n)(*[Cand(c[0], c[1], c[2], c[3], c[4], c[5]) for c in cands])
        out = (Polished * n)()
        if device_ptr is not None:
            src, on_dev = C.c_void_p(device_ptr), 1
        else:
            fft = np.ascontiguousarray(fft, dtype=np.complex64)
            src, on_dev = C.c_void_p(fft.ctypes.data), 0
        self._check(self.L.ab_optimize_cands(self.ptr, C.byref(obs), src, on_dev, arr, n, out),
                    "ab_optimize_cands")
        res = []
        for o in out:
            h = o.numharm
            d = np.array([[getattr(o.derivs[k], f) for f in ("pow", "phs", "dpow", "dphs", "d2pow",
                                                              "d2phs", "locpow")]
                          for k in range(h)])
            res.append(dict(pows=np.array(o.pows[:h]), hirs=np.array(o.hirs[:h]),
                            hizs=np.array(o.hizs[:h]), hiws=np.array(o.hiws[:h]), derivs=d))
        return res

    def realfft(self, series):
        """realfft(data, n, -1) on the device: n/2 complex bins."""
        x = np.ascontiguousarray(series, dtype=np.float32)
        out = np.zeros(x.size // 2, np.complex64)
        self._check(self.L.ab_realfft(self.ptr, x.ctypes.data, x.size, 0, out.ctypes.data, 0),
                    "ab_realfft")
        return out

    def deredden(self, fft, startwidth=6, endwidth=200, endfreq=1e300, T=1.0):
        y = np.ascontiguousarray(fft, dtype=np.complex64).copy()
        self._check(self.L.ab_deredden(self.ptr, y.ctypes.data, y.size, startwidth, endwidth,
                                       endfreq, T, 0), "ab_deredden")
        return y

    def series_to_fft(self, series, dt):
        """accelsearch's .dat input: realfft, then deredden(6, 200, 0.5/dt, n dt)."""
        x = np.ascontiguousarray(series, dtype=np.float32)
        out = np.zeros(x.size // 2, np.complex64)
        self._check(self.L.ab_series_to_fft(self.ptr, x.ctypes.data, x.size, float(dt), 0,
                                            out.ctypes.data, 0), "ab_series_to_fft")
        return out

    def zapbirds(self, fft, N, lobins, hibins, device_ptr=None, numbins=None):
        """-zaplist zapping (ab_zapbirds) of a host spectrum (returns the
        zapped copy) or, with device_ptr, of numbins bins in device memory
        (zapped in place; returns None).  The birdie count zapped is kept in
        self.last_numzapped."""
        lo = np.ascontiguousarray(lobins, dtype=np.float64)
        hi = np.ascontiguousarray(hibins, dtype=np.float64)
        nz = C.c_int()
        if device_ptr is not None:
            self._check(self.L.ab_zapbirds(self.ptr, C.c_void_p(device_ptr), 1, int(numbins),
                                           int(N), lo.ctypes.data, hi.ctypes.data, lo.size,
                                           C.byref(nz)), "ab_zapbirds")
            self.last_numzapped = nz.value
            return None
        y = np.ascontiguousarray(fft, dtype=np.complex64).copy()
        self._check(self.L.ab_zapbirds(self.ptr, y.ctypes.data, 0, y.size, int(N),
                                       lo.ctypes.data, hi.ctypes.data, lo.size, C.byref(nz)),
                    "ab_zapbirds")
        self.last_numzapped = nz.value
        return y

    def dedisperse(self, data, lofreq, chanwidth, dt, nsub, dms, downsamp=1, device_ptr=None,
                   nspec=None, nchan=None, out_ptr=None):
        """Subband dedispersion (ab_dedisperse) of time-major float spectra
        data[nspec][nchan] (channel 0 the lowest frequency); returns
        out[ndm][nspec // downsamp] (or fills out_ptr with device_ptr input)."""
        dmv = np.ascontiguousarray(dms, dtype=np.float64)
        if device_ptr is not None:
            nout = int(nspec) // downsamp
            self._check(self.L.ab_dedisperse(self.ptr, C.c_void_p(device_ptr), 1, int(nspec),
                                             int(nchan), lofreq, chanwidth, dt, nsub,
                                             dmv.ctypes.data, dmv.size, downsamp,
                                             C.c_void_p(out_ptr), 1), "ab_dedisperse")
            return None
        x = np.ascontiguousarray(data, dtype=np.float32)
        nspec, nchan = x.shape
        out = np.zeros((dmv.size, nspec // downsamp), np.float32)
        self._check(self.L.ab_dedisperse(self.ptr, x.ctypes.data, 0, nspec, nchan, lofreq,
                                         chanwidth, dt, nsub, dmv.ctypes.data, dmv.size,
                                         downsamp, out.ctypes.data, 0), "ab_dedisperse")
        return out

    def search_dedispersed(self, data, lofreq, chanwidth, dt, nsub, dms, obs, downsamp=1,
                           device_ptr=None, nspec=None, nchan=None):
        """Dedisperses time-major float spectra data[nspec][nchan] and searches
        every DM trial on the device (ab_search_dedispersed): returns one
        candidate list per DM, each as search() returns it.  obs describes a
        trial: obs_init(make_params((nspec // downsamp) & ~1, dt * downsamp,
        ...))."""
        dmv = np.ascontiguousarray(dms, dtype=np.float64)
        if device_ptr is not None:
            src, on_dev, ns, nc = C.c_void_p(device_ptr), 1, int(nspec), int(nchan)
        else:
            x = np.ascontiguousarray(data, dtype=np.float32)
            ns, nc = x.shape
            src, on_dev = C.c_void_p(x.ctypes.data), 0
        first = (C.c_longlong * (dmv.size + 1))()
        args = (self.ptr, src, on_dev, ns, nc, lofreq, chanwidth, dt, nsub, dmv.ctypes.data,
                dmv.size, downsamp, C.byref(obs))
        cap = 1 << 16
        cands = (Cand * cap)()
        rc = self.L.ab_search_dedispersed(*args, cands, cap, first)
        if rc == -4 and first[dmv.size] > cap:
            # more candidates than the first buffer held: search again into one
            # of the size the first pass counted
            cap = first[dmv.size]
            cands = (Cand * cap)()
            rc = self.L.ab_search_dedispersed(*args, cands, cap, first)
        self._check(rc, "ab_search_dedispersed")
        out = []
        for k in range(dmv.size):
            out.append([(c.power, c.sigma, c.numharm, c.r, c.z, c.w)
                        for c in cands[first[k]:first[k + 1]]])
        return out

    def autotune(self):
        """Measure the correlation cost per transform length on this context's
        device and install it process-wide; returns the table."""
        c = (C.c_double * COST_SLOTS)()
        self._check(self.L.ab_autotune(self.ptr, c, COST_SLOTS), "ab_autotune")
        return list(c)

    def set_corr_path(self, path):
        """CORR_FFT (FP32 FFT correlation, default), CORR_TC_SPLIT_BF16 or
        CORR_TC_SPLIT_FP16 (tensor-core banded contraction, split BF16 or FP16
        operands)."""
        self._check(self.L.ab_ctx_set_corr_path(self.ptr, int(path)), "ab_ctx_set_corr_path")

    # ---- timing -------------------------------------------------------------
    def set_profiling(self, on):
        self.L.ab_ctx_set_profiling(self.ptr, int(on))

    def kernel_times(self):
        """Per kind: 0 templates, 1 prep, 2 correlation, 3 harmonic sum + search
        (device ms); 4 host setup until the last launch is queued, 5 host sort +
        replay, 6 wait for the device and hit read-back (host wall ms); 7
        dedispersion (device ms)."""
        ms = (C.c_double * 8)()
        n = (C.c_longlong * 8)()
        self.L.ab_ctx_kernel_times(self.ptr, ms, n, 8)
        return list(ms), list(n)

    def reset_kernel_times(self):
        self.L.ab_ctx_reset_kernel_times(self.ptr)

    def launch_count(self):
        return self.L.ab_ctx_launch_count(self.ptr)


class CandList:
    """The candidate list search_ffdotpows grows (GSList of accelcand)."""

    def __init__(self):
        self.L = lib()
        self.ptr = self.L.ab_candlist_new()

    def insert(self, power, sigma, numharm, r, z, w):
        return self.L.ab_candlist_insert(self.ptr, power, sigma, numharm, r, z, w)

    def get(self):
        n = self.L.ab_candlist_get(self.ptr, None, 0)
        arr = (Cand * max(n, 1))()
        self.L.ab_candlist_get(self.ptr, arr, n)
        return [(c.power, c.sigma, c.numharm, c.r, c.z, c.w) for c in arr[:n]]

    def set_worklog(self, on, T):
        """Record the .txtcand line of every candidate an insertion adds (T the
        observation's length, s)."""
        if self.L.ab_candlist_set_worklog(self.ptr, int(bool(on)), float(T)):
            raise AccelError("ab_candlist_set_worklog: T must be > 0")

    def worklog(self):
        n = self.L.ab_candlist_worklog(self.ptr, None, 0)
        buf = C.create_string_buffer(n + 1)
        self.L.ab_candlist_worklog(self.ptr, buf, n + 1)
        return buf.raw[:n].decode()

    def __del__(self):
        try:
            self.L.ab_candlist_free(self.ptr)
        except Exception:
            pass


def read_zaplist(path, T, baryv=0.0):
    """get_birdies: (lobins, hibins) arrays of a zap list, sorted by low bin."""
    L = lib()
    n = C.c_int()
    rc = L.ab_read_zaplist(str(path).encode(), float(T), float(baryv), None, None, 0, C.byref(n))
    if rc not in (0, -4):
        raise AccelError(f"ab_read_zaplist: {ERRORS.get(rc, rc)}")
    lo = np.zeros(max(n.value, 1), np.float64)
    hi = np.zeros(max(n.value, 1), np.float64)
    rc = L.ab_read_zaplist(str(path).encode(), float(T), float(baryv), lo.ctypes.data,
                           hi.ctypes.data, n.value, C.byref(n))
    if rc:
        raise AccelError(f"ab_read_zaplist: {ERRORS.get(rc, rc)}")
    return lo[:n.value], hi[:n.value]


def zapbirds_host(fft, N, lobins, hibins):
    """ab_zapbirds_host: the zapped copy of a host spectrum (no GPU)."""
    lo = np.ascontiguousarray(lobins, dtype=np.float64)
    hi = np.ascontiguousarray(hibins, dtype=np.float64)
    y = np.ascontiguousarray(fft, dtype=np.complex64).copy()
    nz = C.c_int()
    rc = lib().ab_zapbirds_host(y.ctypes.data, y.size, int(N), lo.ctypes.data, hi.ctypes.data,
                                lo.size, C.byref(nz))
    if rc:
        raise AccelError(f"ab_zapbirds_host: {ERRORS.get(rc, rc)}")
    return y


def mt19937_output(seed, k):
    return int(lib().ab_mt19937_output(int(seed), int(k)))


def dedisp_delays(nchan, lofreq, chanwidth, dt, nsub, dms, downsamp=1):
    """ab_dedisp_delays: (channel delays [nchan], subband offsets [ndm][nsub])."""
    dmv = np.ascontiguousarray(dms, dtype=np.float64)
    cd = np.zeros(nchan, np.int32)
    off = np.zeros((dmv.size, nsub), np.int32)
    rc = lib().ab_dedisp_delays(nchan, lofreq, chanwidth, dt, nsub, dmv.ctypes.data, dmv.size,
                                downsamp, cd.ctypes.data, off.ctypes.data)
    if rc:
        raise AccelError(f"ab_dedisp_delays: {ERRORS.get(rc, rc)}")
    return cd, off


def candidate_sigma(power, numsum, numtrials):
    return lib().ab_candidate_sigma(float(power), int(numsum), float(numtrials))


def power_for_sigma(sigma, numsum, numtrials):
    return lib().ab_power_for_sigma(float(sigma), int(numsum), float(numtrials))


def sort_cands(cands):
    n = len(cands)
    arr = (Cand * max(n, 1))(*[Cand(*c) for c in cands])
    lib().ab_sort_cands(arr, n)
    return [(c.power, c.sigma, c.numharm, c.r, c.z, c.w) for c in arr[:n]]


def eliminate_harmonics(cands):
    n = len(cands)
    arr = (Cand * max(n, 1))(*[Cand(*c) for c in cands])
    m = lib().ab_eliminate_harmonics(arr, n)
    return [(c.power, c.sigma, c.numharm, c.r, c.z, c.w) for c in arr[:m]]


class AccelSearch:
    """accelsearch for one spectrum: options as on the command line."""

    def __init__(self, zmax=200, wmax=None, numharm=8, sigma=2.0, flo=1.0, fhi=10000.0,
                 rlo=None, rhi=None, inmem=False, photon=None, lobin=0, locpow=False,
                 noharmpolish=False, device=0, ctx=None):
        self.opts = dict(zmax=zmax, wmax=wmax, numharm=numharm, sigma=sigma, flo=flo, fhi=fhi,
                         rlo=rlo, rhi=rhi, inmem=inmem, photon=photon, lobin=lobin, locpow=locpow,
                         noharmpolish=noharmpolish)
        self.ctx = ctx or Context(device)

    def obs(self, N, dt, numbins=None):
        return obs_init(make_params(N, dt, numbins, **self.opts))

    def __call__(self, fft, N, dt):
        fft = np.ascontiguousarray(fft, dtype=np.complex64)
        obs = self.obs(N, dt, fft.size)
        return self.ctx.search(obs, fft)

    def run_series(self, series, dt, zaplist=None, baryv=0.0, harmremove=True, candfile=None,
                   rootname=None):
        """accelsearch on a .dat time series (src/accel_utils.c:1507-1563 and
        src/accelsearch.c:87-110): realfft and deredden on the device, the
        -zaplist birdies zapped (zaplist: a zap-list file) in the device
        spectrum, then run() with the reference's .dat conventions (no
        .txtcand).  Returns run()'s dict."""
        x = np.ascontiguousarray(series, dtype=np.float32)
        N = x.size
        fft = self.ctx.series_to_fft(x, dt)
        if zaplist is not None:
            lo, hi = read_zaplist(zaplist, N * dt, baryv)
            fft = self.ctx.zapbirds(fft, N, lo, hi)
        return self.run(fft, N, dt, harmremove=harmremove, candfile=candfile, rootname=rootname,
                        dat_input=True)

    def run(self, fft, N, dt, harmremove=True, candfile=None, rootname=None, dat_input=False):
        """The whole of src/accelsearch.c:155-284 for one spectrum: the search,
        sort_accelcands, eliminate_harmonics (numharm > 1 unless harmremove
        is False, as -noharmremove), optimize_accelcand of every candidate on
        the device, and the fundamentals' .cand records (written to candfile
        when given).  With rootname, the reference's output files too:
        <rootname>_ACCEL_<zmax>[_JERK_<wmax>] (text, with <rootname>.inf
        appended when it exists), its .cand and the .txtcand work file, one
        line per candidate insertion during the search (src/accel_utils.c:
        1443-1447, 1667-1685); with no candidates only the .txtcand, as the
        reference.  Returns dict(cands, polished, props, obs)."""
        fft = np.ascontiguousarray(fft, dtype=np.complex64)
        obs = self.obs(N, dt, fft.size)
        log = bool(rootname) and not dat_input      # .dat input: no .txtcand
        if log:
            self.ctx.set_worklog(True)
        try:
            cands = self.ctx.search(obs, fft)
            worklog = self.ctx.last_worklog() if log else ""
        finally:
            if log:
                self.ctx.set_worklog(False)
        polished, props = [], []
        if cands:
            cands = sort_cands(cands)
            if self.opts["numharm"] > 1 and harmremove:
                cands = eliminate_harmonics(cands)
            polished = self.ctx.optimize_cands(obs, fft, cands)
            props = cand_props(cands, polished)
            if candfile:
                write_candfile(candfile, props)
        if rootname:
            names = accel_filenames(rootname, obs)
            if not dat_input:
                with open(names["txtcand"], "w") as f:
                    f.write(worklog)
            if cands:
                inf = rootname + ".inf"
                write_accelfile(names["accel"], obs, cands, polished,
                                inf if os.path.exists(inf) else None)
                write_candfile(names["cand"], props)
        return dict(cands=cands, polished=polished, props=props, obs=obs)
