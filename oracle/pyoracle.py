"""ctypes binding of the CPU oracle (oracle/accel_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py.  The product (presto_b200) never imports it.
"""
import ctypes as C  # noqa: N812
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


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


class FFDot(C.Structure):
    _fields_ = [("rlo", C.c_longlong), ("zlo", C.c_int), ("wlo", C.c_int),
                ("numrs", C.c_int), ("numzs", C.c_int), ("numws", C.c_int),
                ("powers", C.POINTER(C.c_float)),
                ("rinds", C.POINTER(C.c_ushort)), ("zinds", C.POINTER(C.c_ushort))]


class Cand(C.Structure):
    _fields_ = [("power", C.c_float), ("sigma", C.c_float), ("numharm", C.c_int),
                ("r", C.c_double), ("z", C.c_double), ("w", C.c_double)]


class Hit(C.Structure):
    _fields_ = [("block", C.c_longlong), ("stage", C.c_int), ("wi", C.c_int),
                ("zi", C.c_int), ("ri", C.c_int), ("power", C.c_float)]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_libs = {}


def lib(prec=64):
    if prec not in _libs:
        path = os.path.join(HERE, f"liboracle{prec}.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp = C.c_void_p
        L.orc_obs_init.argtypes = [C.POINTER(Params), C.POINTER(Obs)]
        L.orc_bank_create.restype = vp
        L.orc_bank_create.argtypes = [C.POINTER(Obs), C.c_int, C.c_int]
        L.orc_bank_free.argtypes = [vp]
        L.orc_bank_info.argtypes = [vp] + [C.POINTER(C.c_int)] * 6
        L.orc_bank_kernel.argtypes = [vp, C.c_int, C.c_int, vp]
        L.orc_subharm_fderivs_vol.argtypes = [C.POINTER(Obs), vp, C.c_int, C.c_int,
                                              C.c_double, C.c_double, vp, C.POINTER(FFDot)]
        L.orc_ffdot_free.argtypes = [C.POINTER(FFDot)]
        L.orc_add_ffdotpows.argtypes = [C.POINTER(FFDot), C.POINTER(FFDot), C.c_int, C.c_int]
        L.orc_fund_to_ffdotplane.argtypes = [C.POINTER(FFDot), C.POINTER(Obs), vp]
        L.orc_inmem_add_ffdotpows.argtypes = [C.POINTER(FFDot), C.POINTER(Obs), vp,
                                              C.c_int, C.c_int]
        for name in ("orc_chi2_logp", "orc_chisq_q", "orc_chisq_qinv"):
            getattr(L, name).restype = C.c_double
            getattr(L, name).argtypes = [C.c_double, C.c_double]
        for name in ("orc_equivalent_gaussian_sigma", "orc_gauss_q", "orc_gauss_qinv"):
            getattr(L, name).restype = C.c_double
            getattr(L, name).argtypes = [C.c_double]
        for name in ("orc_candidate_sigma", "orc_power_for_sigma"):
            getattr(L, name).restype = C.c_double
            getattr(L, name).argtypes = [C.c_double, C.c_int, C.c_double]
        L.orc_median.restype = C.c_float
        L.orc_median.argtypes = [vp, C.c_int]
        L.orc_fresnel.argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_gen_r_response.argtypes = [C.c_double, C.c_int, C.c_int, vp]
        L.orc_gen_z_response.argtypes = [C.c_double, C.c_int, C.c_double, C.c_int, vp]
        L.orc_gen_w_response.argtypes = [C.c_double, C.c_int, C.c_double, C.c_double,
                                         C.c_int, vp]
        for name in ("orc_z_resp_halfwidth",):
            getattr(L, name).argtypes = [C.c_double]
        L.orc_w_resp_halfwidth.argtypes = [C.c_double, C.c_double]
        L.orc_next_good_fftlen.argtypes = [C.c_int]
        L.orc_fftlen_from_kernwidth.argtypes = [C.c_int]
        L.orc_calc_required_r.restype = C.c_double
        L.orc_calc_required_r.argtypes = [C.c_double, C.c_double]
        L.orc_calc_required_z.argtypes = [C.c_double, C.c_double]
        L.orc_calc_required_w.argtypes = [C.c_double, C.c_double]
        L.orc_accelsearch.restype = C.c_longlong
        L.orc_accelsearch.argtypes = [C.POINTER(Params), vp, C.c_int, C.c_longlong,
                                      C.c_longlong, C.POINTER(Cand), C.c_longlong,
                                      C.POINTER(Hit), C.c_longlong, C.POINTER(C.c_longlong),
                                      C.POINTER(C.c_longlong)]
        L.orc_list_new.restype = vp
        L.orc_list_free.argtypes = [vp]
        L.orc_list_insert.argtypes = [vp, C.c_float, C.c_float, C.c_int,
                                      C.c_double, C.c_double, C.c_double]
        L.orc_list_get.restype = C.c_longlong
        L.orc_list_get.argtypes = [vp, C.POINTER(Cand), C.c_longlong]
        L.orc_search_ffdotpows.argtypes = [C.POINTER(FFDot), C.c_int, C.POINTER(Obs), vp,
                                           C.c_longlong, C.POINTER(Hit), C.c_longlong,
                                           C.POINTER(C.c_longlong)]
        _libs[prec] = L
    return _libs[prec]


def make_params(N, dt, numbins, zmax=200, wmax=None, numharm=8, sigma=2.0,
                flo=1.0, fhi=10000.0, inmem=False, rlo=None, rhi=None, nph=0.0, lobin=0,
                locpow=False, noharmpolish=False):
    """Mirror of the accelsearch command line defaults (src/accelsearch_cmd.c:22-61)."""
    p = Params()
    p.N, p.dt, p.numbins = N, dt, numbins
    p.zmax = zmax
    p.wmax = 0 if wmax is None else wmax
    p.wmaxP = 0 if wmax is None else 1
    p.numharm, p.sigma = numharm, sigma
    p.flo, p.fhi = flo, fhi
    p.floP = 1 if rlo is None else 0
    p.fhiP = 1 if rhi is None else 0
    p.rlo = rlo or 0.0
    p.rhi = rhi or 0.0
    p.rloP = 0 if rlo is None else 1
    p.rhiP = 0 if rhi is None else 1
    p.lobin, p.inmemP, p.nph = lobin, int(inmem), nph
    p.locpowP = int(bool(locpow))
    p.noharmpolishP = int(bool(noharmpolish))
    return p


def obs_init(p, prec=64):
    o = Obs()
    rc = lib(prec).orc_obs_init(C.byref(p), C.byref(o))
    if rc:
        raise ValueError(f"orc_obs_init failed: {rc}")
    return o


def response(kind, numbetween, numkern, z=0.0, w=0.0, roffset=0.0):
    L = lib(64)
    out = np.zeros(numkern, np.complex64)
    if kind == "r":
        rc = L.orc_gen_r_response(roffset, numbetween, numkern, out.ctypes.data)
    elif kind == "z":
        rc = L.orc_gen_z_response(roffset, numbetween, z, numkern, out.ctypes.data)
    else:
        rc = L.orc_gen_w_response(roffset, numbetween, z, w, numkern, out.ctypes.data)
    if rc:
        raise ValueError("bad response arguments")
    return out


def fresnel(x):
    s, c = C.c_double(), C.c_double()
    lib(64).orc_fresnel(float(x), C.byref(s), C.byref(c))
    return s.value, c.value


class Bank:
    def __init__(self, obs, numharm, harmnum, prec=64):
        self.L = lib(prec)
        self.ptr = self.L.orc_bank_create(C.byref(obs), numharm, harmnum)
        vals = [C.c_int() for _ in range(6)]
        self.L.orc_bank_info(self.ptr, *[C.byref(v) for v in vals])
        (self.zmax, self.wmax, self.nz, self.nw, self.fftlen, self.halfwidth) = [v.value for v in vals]

    def kernel(self, wi, zi):
        out = np.zeros(self.fftlen, np.complex64)
        self.L.orc_bank_kernel(self.ptr, wi, zi, out.ctypes.data)
        return out

    def __del__(self):
        try:
            self.L.orc_bank_free(self.ptr)
        except Exception:
            pass


def subharm_fderivs_vol(obs, fft, numharm, harmnum, fullrlo, fullrhi, bank, prec=64):
    """Returns (meta dict, powers[w][z][r] ndarray, rinds, zinds)."""
    L = lib(prec)
    f = FFDot()
    L.orc_subharm_fderivs_vol(C.byref(obs), fft.ctypes.data, numharm, harmnum,
                              fullrlo, fullrhi, bank.ptr, C.byref(f))
    n = f.numws * f.numzs * f.numrs
    pw = np.ctypeslib.as_array(f.powers, shape=(n,)).copy().reshape(f.numws, f.numzs, f.numrs)
    rinds = zinds = None
    if numharm > 1 and not obs.inmem:
        rinds = np.ctypeslib.as_array(f.rinds, shape=(obs.corr_uselen,)).copy()
        zinds = np.ctypeslib.as_array(f.zinds, shape=(obs.numz,)).copy()
    meta = dict(rlo=f.rlo, zlo=f.zlo, wlo=f.wlo, numrs=f.numrs, numzs=f.numzs, numws=f.numws)
    L.orc_ffdot_free(C.byref(f))
    return meta, pw, rinds, zinds


def accelsearch(p, fft, nthreads=1, first_block=0, max_blocks=-1, maxcands=100000,
                maxhits=2000000, prec=64):
    L = lib(prec)
    cands = (Cand * maxcands)()
    hits = (Hit * maxhits)()
    nh, nb = C.c_longlong(), C.c_longlong()
    fft = np.ascontiguousarray(fft, dtype=np.complex64)
    nc = L.orc_accelsearch(C.byref(p), fft.ctypes.data, nthreads, first_block, max_blocks,
                           cands, maxcands, hits, maxhits, C.byref(nh), C.byref(nb))
    if nc < 0:
        raise RuntimeError("orc_accelsearch failed")
    cl = [(c.power, c.sigma, c.numharm, c.r, c.z, c.w) for c in cands[:min(nc, maxcands)]]
    hl = [(h.block, h.stage, h.wi, h.zi, h.ri, h.power) for h in hits[:min(nh.value, maxhits)]]
    return cl, hl, nb.value


def ref_fresnel_lib():
    """The reference's own fresnl.c built by build_ref.sh, or None."""
    path = os.path.join(HERE, "_ref", "libref_fresnl.so")
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    L.fresnl.argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.fresnl.restype = C.c_int
    return L


# ---- candidate polishing (polish_oracle.c) --------------------------------
MAX_HARM = 32


class RDerivs(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("pow", "phs", "dpow", "dphs", "d2pow", "d2phs",
                                         "locpow")]


class FourierProps(C.Structure):
    _fields_ = [("r", C.c_double), ("rerr", C.c_float), ("z", C.c_double), ("zerr", C.c_float),
                ("w", C.c_double), ("werr", C.c_float)] + \
               [(n, C.c_float) for n in ("pow", "powerr", "sig", "rawpow", "phs", "phserr", "cen",
                                         "cenerr", "pur", "purerr", "locpow")]


def _polish_lib():
    L = lib(64)
    if not getattr(L, "_polish_ready", False):
        d, i, vp = C.c_double, C.c_int, C.c_void_p
        L.orc_rzw_interp.argtypes = [vp, C.c_long, d, d, d, i, vp]
        L.orc_get_localpower3d.restype = d
        L.orc_get_localpower3d.argtypes = [vp, C.c_long, d, d, d]
        L.orc_get_derivs3d.argtypes = [vp, C.c_long, d, d, d, d, C.POINTER(RDerivs)]
        L.orc_calc_props.argtypes = [C.POINTER(RDerivs), d, d, d, C.POINTER(FourierProps)]
        L.orc_max_rz_arr.restype = d
        L.orc_max_rz_arr.argtypes = [vp, C.c_long, d, d, C.POINTER(d), C.POINTER(d),
                                     C.POINTER(RDerivs)]
        L.orc_max_rz_arr_harmonics.argtypes = [vp, C.c_long, i, d, d, C.POINTER(d), C.POINTER(d),
                                               C.POINTER(RDerivs), C.POINTER(d)]
        L.orc_optimize_cands.argtypes = [vp, C.c_longlong, C.c_longlong, i, vp, vp, vp, vp, vp,
                                         vp, vp, i]
        L.orc_z_resp_halfwidth_acc.argtypes = [d, i]
        L.orc_w_resp_halfwidth_acc.argtypes = [d, d, i]
        L.orc_max_rzw_arr.restype = d
        L.orc_max_rzw_arr.argtypes = [vp, C.c_long, d, d, d, C.POINTER(d), C.POINTER(d),
                                      C.POINTER(d), C.POINTER(RDerivs)]
        L.orc_max_rzw_arr_harmonics.argtypes = [vp, C.c_long, i, d, d, d, C.POINTER(d),
                                                C.POINTER(d), C.POINTER(d), C.POINTER(RDerivs),
                                                C.POINTER(d)]
        L.orc_optimize_cands_w.argtypes = [vp, C.c_longlong, C.c_longlong, i, i, vp, vp, vp, vp,
                                           vp, vp, vp, vp, vp, i]
        L.orc_rzw_vol_point.argtypes = [vp, C.c_long, C.c_long, i, C.c_long, vp, i, vp]
        L._polish_ready = True
    return L


def rz_interp(data, r, z, kern_half_width, w=0.0):
    data = np.ascontiguousarray(data, dtype=np.complex64)
    a = np.zeros(1, np.complex64)
    _polish_lib().orc_rzw_interp(data.ctypes.data, data.size, r, z, w, kern_half_width,
                                 a.ctypes.data)
    return complex(a[0])


def max_rz_arr(data, r, z):
    """(power, rout, zout, rderivs) of the single-harmonic optimiser."""
    data = np.ascontiguousarray(data, dtype=np.complex64)
    ro, zo, rd = C.c_double(), C.c_double(), RDerivs()
    p = _polish_lib().orc_max_rz_arr(data.ctypes.data, data.size, r, z, C.byref(ro), C.byref(zo),
                                      C.byref(rd))
    return p, ro.value, zo.value, rd


def max_rz_arr_harmonics(data, r, z, numharm):
    """(rout, zout, [rderivs per harmonic], [raw power per harmonic])."""
    data = np.ascontiguousarray(data, dtype=np.complex64)
    ro, zo = C.c_double(), C.c_double()
    rds = (RDerivs * numharm)()
    pw = (C.c_double * numharm)()
    _polish_lib().orc_max_rz_arr_harmonics(data.ctypes.data, data.size, numharm, r, z,
                                           C.byref(ro), C.byref(zo), rds, pw)
    return ro.value, zo.value, list(rds), list(pw)


def max_rzw_arr(data, r, z, w):
    """(power, rout, zout, wout, rderivs) of the single-harmonic jerk maximiser."""
    data = np.ascontiguousarray(data, dtype=np.complex64)
    ro, zo, wo, rd = C.c_double(), C.c_double(), C.c_double(), RDerivs()
    p = _polish_lib().orc_max_rzw_arr(data.ctypes.data, data.size, r, z, w, C.byref(ro),
                                       C.byref(zo), C.byref(wo), C.byref(rd))
    return p, ro.value, zo.value, wo.value, rd


def max_rzw_arr_harmonics(data, r, z, w, numharm):
    """(rout, zout, wout, [rderivs per harmonic], [power per harmonic])."""
    data = np.ascontiguousarray(data, dtype=np.complex64)
    ro, zo, wo = C.c_double(), C.c_double(), C.c_double()
    rds = (RDerivs * numharm)()
    pw = (C.c_double * numharm)()
    _polish_lib().orc_max_rzw_arr_harmonics(data.ctypes.data, data.size, numharm, r, z, w,
                                            C.byref(ro), C.byref(zo), C.byref(wo), rds, pw)
    return ro.value, zo.value, wo.value, list(rds), list(pw)


def rzw_vol_point(data, beginbin, numbetween, j, resp):
    """One output of corr_rzw_vol's volume as the direct correlation sum."""
    data = np.ascontiguousarray(data, dtype=np.complex64)
    resp = np.ascontiguousarray(resp, dtype=np.complex64)
    a = np.zeros(1, np.complex64)
    _polish_lib().orc_rzw_vol_point(data.ctypes.data, data.size, int(beginbin), int(numbetween),
                                    int(j), resp.ctypes.data, resp.size, a.ctypes.data)
    return complex(a[0])


def w_resp_halfwidth_acc(z, w, highacc=False):
    return _polish_lib().orc_w_resp_halfwidth_acc(float(z), float(w), int(bool(highacc)))


def optimize_cands_w(fft, lobin, cands, jerk, nthreads=1):
    """optimize_accelcand for (numharm, r, z, w) candidates of an acceleration
    (jerk False) or jerk (jerk True) search: per candidate a dict of pows,
    hirs, hizs, hiws (numharm entries) and the derivs array."""
    fft = np.ascontiguousarray(fft, dtype=np.complex64)
    n = len(cands)
    nh = np.array([c[0] for c in cands], np.int32)
    r = np.array([c[1] for c in cands], np.float64)
    z = np.array([c[2] for c in cands], np.float64)
    w = np.array([c[3] if len(c) > 3 else 0.0 for c in cands], np.float64)
    pows, hirs, hizs, hiws = (np.zeros((n, MAX_HARM)) for _ in range(4))
    der = np.zeros((n, MAX_HARM, 7))
    rc = _polish_lib().orc_optimize_cands_w(fft.ctypes.data, fft.size, int(lobin), n, int(bool(jerk)),
                                            nh.ctypes.data, r.ctypes.data, z.ctypes.data,
                                            w.ctypes.data, pows.ctypes.data, hirs.ctypes.data,
                                            hizs.ctypes.data, hiws.ctypes.data, der.ctypes.data,
                                            int(nthreads))
    if rc:
        raise RuntimeError("orc_optimize_cands_w failed")
    return [dict(pows=pows[k, :nh[k]], hirs=hirs[k, :nh[k]], hizs=hizs[k, :nh[k]],
                 hiws=hiws[k, :nh[k]], derivs=der[k, :nh[k]]) for k in range(n)]


def optimize_cands(fft, lobin, cands, nthreads=1):
    """optimize_accelcand for (numharm, r, z) candidates: per candidate a dict
    of pows, hirs, hizs (numharm entries) and the derivs array."""
    fft = np.ascontiguousarray(fft, dtype=np.complex64)
    n = len(cands)
    nh = np.array([c[0] for c in cands], np.int32)
    r = np.array([c[1] for c in cands], np.float64)
    z = np.array([c[2] for c in cands], np.float64)
    pows = np.zeros((n, MAX_HARM))
    hirs = np.zeros((n, MAX_HARM))
    hizs = np.zeros((n, MAX_HARM))
    der = np.zeros((n, MAX_HARM, 7))
    rc = _polish_lib().orc_optimize_cands(fft.ctypes.data, fft.size, int(lobin), n, nh.ctypes.data,
                                          r.ctypes.data, z.ctypes.data, pows.ctypes.data,
                                          hirs.ctypes.data, hizs.ctypes.data, der.ctypes.data,
                                          int(nthreads))
    if rc:
        raise RuntimeError("orc_optimize_cands failed")
    return [dict(pows=pows[k, :nh[k]], hirs=hirs[k, :nh[k]], hizs=hizs[k, :nh[k]],
                 derivs=der[k, :nh[k]]) for k in range(n)]


# ---- time-series input path (series_oracle.c) ------------------------------
def _series_lib():
    L = lib(64)
    if not getattr(L, "_series_ready", False):
        L.orc_realfft_forward.argtypes = [C.c_void_p, C.c_long]
        L.orc_deredden.restype = C.c_long
        L.orc_deredden.argtypes = [C.c_void_p, C.c_long, C.c_int, C.c_int, C.c_double, C.c_double]
        L.orc_invsqrtf.restype = C.c_float
        L.orc_invsqrtf.argtypes = [C.c_float]
        L._series_ready = True
    return L


def loc_pow(powers):
    """corr_loc_pow (src/corr_routines.c:309-366) restated exactly."""
    pw = np.ascontiguousarray(powers, dtype=np.float32)
    out = np.zeros_like(pw)
    L = _series_lib()
    L.orc_loc_pow.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    L.orc_loc_pow(pw.ctypes.data, pw.size, out.ctypes.data)
    return out


def realfft(series):
    """realfft(data, n, -1): n/2 complex bins, bin 0 = (DC, Nyquist)."""
    x = np.ascontiguousarray(series, dtype=np.float32).copy()
    if _series_lib().orc_realfft_forward(x.ctypes.data, x.size):
        raise ValueError("realfft needs a length divisible by 4")
    return x.view(np.complex64)


def deredden(fft, startwidth=6, endwidth=200, endfreq=None, T=1.0):
    """deredden on a copy of fft (accelsearch uses 6, 200, Nyquist, N dt)."""
    y = np.ascontiguousarray(fft, dtype=np.complex64).copy()
    if endfreq is None:
        endfreq = 1e300
    n = _series_lib().orc_deredden(y.ctypes.data, y.size, startwidth, endwidth, endfreq, T)
    if n < 0:
        raise ValueError("deredden failed")
    return y
