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
        L.orc_accelsearch_sample.restype = C.c_longlong
        L.orc_accelsearch_sample.argtypes = [C.POINTER(Params), vp, C.c_int, C.c_longlong,
                                             C.c_longlong, C.c_longlong, vp, C.c_longlong, vp,
                                             C.c_longlong, C.POINTER(C.c_longlong),
                                             C.POINTER(C.c_longlong)]
        L.orc_last_fft_share.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
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


def accelsearch_sample(p, fft, nthreads, first_block, max_blocks, block_stride, prec=32,
                       libpath=None, loop_threads=0):
    """Times a search over every block_stride-th block from first_block
    (max_blocks of them, hits and candidates not kept): returns (blocks done,
    template-bank s, block-loop s, FFT thread-s, loop thread-s).  libpath
    selects another build of the same oracle (e.g. one compiled with
    -march=native); loop_threads > 0 runs the block loop on that many threads
    (the template banks on nthreads)."""
    L = lib(prec) if libpath is None else _lib_at(libpath)
    nb = C.c_longlong()
    fft = np.ascontiguousarray(fft, dtype=np.complex64)
    L.orc_set_loop_threads(int(loop_threads))
    try:
        rc = L.orc_accelsearch_sample(C.byref(p), fft.ctypes.data, nthreads, first_block,
                                      max_blocks, block_stride, None, 0, None, 0, None,
                                      C.byref(nb))
    finally:
        L.orc_set_loop_threads(0)
    if rc < 0:
        raise RuntimeError("orc_accelsearch_sample failed")
    a, b = C.c_double(), C.c_double()
    L.orc_last_timing(C.byref(a), C.byref(b))
    f, t = C.c_double(), C.c_double()
    L.orc_last_fft_share(C.byref(f), C.byref(t))
    return nb.value, a.value, b.value, f.value, t.value


def _lib_at(path):
    if path not in _libs:
        L = C.CDLL(path)
        vp = C.c_void_p
        L.orc_accelsearch_sample.restype = C.c_longlong
        L.orc_accelsearch_sample.argtypes = [C.POINTER(Params), vp, C.c_int, C.c_longlong,
                                             C.c_longlong, C.c_longlong, vp, C.c_longlong, vp,
                                             C.c_longlong, C.POINTER(C.c_longlong),
                                             C.POINTER(C.c_longlong)]
        L.orc_last_timing.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_last_fft_share.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _libs[path] = L
    return _libs[path]


def build_native():
    """liboracle32n.so: the FP32 oracle compiled with -march=native for the
    host it runs on (the reference's documented 1.5-2x build knob); None when
    the compiler refuses."""
    # always rebuilt (-B): a copy built on another host may use instructions
    # this CPU lacks
    r = subprocess.run(["make", "-s", "-B", "-C", HERE, "native"], capture_output=True, text=True)
    path = os.path.join(HERE, "liboracle32n.so")
    return path if r.returncode == 0 and os.path.exists(path) else None


def search_counts(obs):
    """Blocks and f-fdot cells of one search from the oracle's own geometry:
    the main loop's block count (startr from rlo in steps of rstep while
    startr + rstep < highestbin, src/accelsearch.c:187-189) and cells =
    numrs x numz x max(numw, 1) per block per harmonic stage."""
    nb, startr = 0, float(obs.rlo)
    while startr + obs.rstep < obs.highestbin:
        nb += 1
        startr += obs.rstep
    cells = nb * obs.corr_uselen * obs.numz * max(obs.numw, 1) * obs.numharmstages
    return dict(blocks=nb, cells=cells)


def last_timing(prec=64):
    """(template-bank seconds, block-loop seconds) of the last accelsearch."""
    L = lib(prec)
    a, b = C.c_double(), C.c_double()
    L.orc_last_timing(C.byref(a), C.byref(b))
    return a.value, b.value


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


def ref_polish_lib():
    """The reference's src/characteristics.c, rzinterp.c, rzwinterp.c,
    responses.c, fresnl.c, vectors.c and the libpresto files they call
    (realfft, fftwcall), built by build_ref.sh against the FFTW / GSL stand-ins
    of oracle/refshim/, or None.  Its functions exit() on arguments the
    reference rejects: call them with valid ones only."""
    path = os.path.join(HERE, "_ref", "libref_polish.so")
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    d, i, vp = C.c_double, C.c_int, C.c_void_p
    L.gen_r_response.restype = vp
    L.gen_r_response.argtypes = [d, i, i]
    L.gen_z_response.restype = vp
    L.gen_z_response.argtypes = [d, i, d, i]
    L.gen_w_response.restype = vp
    L.gen_w_response.argtypes = [d, i, d, d, i]
    L.vect_free.argtypes = [vp]
    L.z_resp_halfwidth.argtypes = [d, i]
    L.w_resp_halfwidth.argtypes = [d, d, i]
    L.rz_interp.argtypes = [vp, C.c_long, d, d, i, vp]
    L.rzw_interp.argtypes = [vp, C.c_long, d, d, d, i, vp]
    L.get_localpower3d.restype = d
    L.get_localpower3d.argtypes = [vp, C.c_long, d, d, d]
    L.get_derivs3d.argtypes = [vp, C.c_long, d, d, d, d, C.POINTER(RDerivs)]
    L.calc_props.argtypes = [RDerivs, d, d, d, C.POINTER(FourierProps)]
    L.calc_rzwerrs.argtypes = [C.c_void_p, d, C.c_void_p]
    return L


def ref_accel_lib():
    """oracle/refdrv.c over the reference's own objects (build_ref.sh): its
    create_accelobs / create_subharminfos / subharm_fderivs_vol, or None."""
    path = os.path.join(HERE, "_ref", "libref_accel.so")
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    L.refdrv_open.argtypes = [C.c_int, C.POINTER(C.c_char_p)]
    L.refdrv_geometry.argtypes = [C.POINTER(C.c_double)]
    L.refdrv_plane.restype = C.c_longlong
    L.refdrv_plane.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p,
                               C.c_longlong, C.POINTER(C.c_longlong)]
    return L


def ref_plane(L, numharm, harmnum, lo, hi):
    """(meta dict, powers [numws][numzs][numrs]) of the reference's
    subharm_fderivs_vol for the search refdrv_open set up."""
    meta = (C.c_longlong * 6)()
    n = L.refdrv_plane(numharm, harmnum, lo, hi, None, 0, meta)
    out = np.zeros(n, np.float32)
    L.refdrv_plane(numharm, harmnum, lo, hi, out.ctypes.data, n, meta)
    m = dict(zip(("rlo", "zlo", "wlo", "numrs", "numzs", "numws"), [int(v) for v in meta]))
    return m, out.reshape(m["numws"], m["numzs"], m["numrs"])


def ref_response(L, kind, numbetween, numkern, z=0.0, w=0.0, roffset=0.0):
    """gen_r/z/w_response of the reference build, copied out and freed."""
    if kind == "r":
        p = L.gen_r_response(roffset, numbetween, numkern)
    elif kind == "z":
        p = L.gen_z_response(roffset, numbetween, z, numkern)
    else:
        p = L.gen_w_response(roffset, numbetween, z, w, numkern)
    out = np.ctypeslib.as_array((C.c_float * (2 * numkern)).from_address(p)).copy()
    L.vect_free(p)
    return out.view(np.complex64)


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
        raise ValueError("realfft needs an even length")
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


# ---- the ACCEL text candidate file ------------------------------------------
# output_fundamentals / output_harmonics (src/accel_utils.c:666-966),
# compare_rzw_cands (src/accel_utils.c:105-134), center_string
# (src/accel_utils.c:629-643) and nice_output_1 / nice_output_2
# (src/output.c:6-210), restated in Python.  Python's % operator formats
# these conversions as C's printf does and math.* calls the C library.
import math  # noqa: E402

DBLCORRECT = 1e-14
SOL = 299792458.0


class RzwErrs(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("p", "pd", "pdd", "f", "fd", "fdd")] + \
               [(n, C.c_float) for n in ("perr", "pderr", "pdderr", "ferr", "fderr", "fdderr")]


def ref_output_lib():
    """The reference's own src/output.c built by build_ref.sh, or None."""
    path = os.path.join(HERE, "_ref", "libref_output.so")
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    for f in (L.nice_output_1, L.nice_output_2):
        f.argtypes = [C.c_char_p, C.c_double, C.c_double, C.c_int]
        f.restype = C.c_int
    return L


def _cint(x):
    """C's (int) of a double on x86-64: truncation, INT_MIN when out of range."""
    t = int(x)
    return t if -2 ** 31 <= t < 2 ** 31 else -2 ** 31


def _p(prec):
    return prec if prec >= 0 else 6          # C: a negative '*' precision is omitted


def _fin(s, length):
    return s if length == 0 else "%*s" % (length, s)


def nice_output_1(val, err, length=0):
    """val(err), one error digit (src/output.c:6-111)."""
    ee = 0 if abs(err) == 0.0 else math.floor(math.log10(abs(err)))
    ev = _cint(math.floor(abs(err) * math.pow(10.0, -ee) + DBLCORRECT + 0.5))
    if ev == 10:
        ev, ee = 1, ee + 1
    rv = math.pow(10.0, ee) * math.floor(val * math.pow(10.0, -ee) + 0.5)
    nint = 1 if abs(val) == 0.0 else (math.ceil(math.log10(abs(val))) or 1)
    nfrac = -ee
    prec = nint + nfrac
    oexp = 0 if abs(rv) == 0.0 else math.floor(math.log10(abs(rv)))
    mant = rv * math.pow(10.0, -oexp)
    if abs(1.0 - mant) < DBLCORRECT or abs(-1.0 - mant) < DBLCORRECT:
        prec += 1
    sm = -abs(mant) if rv < 0.0 else abs(mant)
    if oexp >= 0 and ee > 0 and oexp > ee:
        s = "% .*f(%d)x10^%d" % (_p(prec - 1), sm, ev, oexp)
    elif oexp >= 0 and ee > 0 and oexp == ee:
        s = "% d(%d)x10^%d" % (_cint(sm), ev, oexp)
    elif oexp < -4 and oexp >= ee:
        s = "% .*f(%d)x10^%d" % (_p(prec - 1), sm, ev, oexp)
    elif oexp < ee and ee != 0:
        s = "% d(%d)x10^%d" % (_cint(sm + DBLCORRECT), ev, ee)
    elif nfrac == 0 and abs(rv) < 1.0e-15:
        s = "% d(%d)" % (_cint(abs(rv)), ev)
    elif abs(rv) <= DBLCORRECT and ee < -5:
        s = "0.0(%d)x10^%d" % (ev, ee + 1)
    else:
        s = "% .*f(%d)" % (_p(nfrac), rv, ev)
    return _fin(s, length)


def nice_output_2(val, err, length=0):
    """val(err), two error digits (src/output.c:114-210); None where the
    reference exits."""
    ee = 0 if abs(err) == 0.0 else math.floor(math.log10(abs(err)))
    ev = _cint(math.floor(abs(err) * math.pow(10.0, -ee + 1) + DBLCORRECT + 0.5))
    if ev == 100:
        ev, ee = 10, ee + 1
    rv = math.pow(10.0, ee - 1) * math.floor(val * math.pow(10.0, -ee + 1) + 0.5)
    oexp = 0 if rv == 0.0 else math.floor(math.log10(abs(rv)))
    vexp = 0 if val == 0.0 else math.floor(math.log10(abs(val)))
    mant = rv * math.pow(10.0, -oexp)
    hi, lo = ev // 10, ev % 10
    if oexp < -4:
        k = oexp - ee + 1
        if k < 2:
            m, x = (mant / 10, oexp + 1) if k == 0 else (mant, oexp)
            s = "% .1f(%d.%d)x10^%d" % (m, hi, lo, x)
        else:
            s = "% .*f(%.2d)x10^%d" % (k, mant, ev, oexp)
    elif ee - vexp > 1 and ee not in (0, 1):
        s = "0.0(%d.%d)x10^%d" % (hi, lo, ee)
    elif ee == 0:
        s = "% .1f(%d.%d)" % (abs(rv) if abs(rv) < 0.1 else rv, hi, lo)
    elif ee < 0:
        if abs(rv) * math.pow(10.0, -ee + 1) < 0.1:
            rv = abs(rv)
        if abs(rv) <= DBLCORRECT and ee < -4:
            s = "0.0(%d.%d)x10^%d" % (hi, lo, ee)
        else:
            s = "% .*f(%.2d)" % (-ee + 1, rv, ev)
    elif ee == oexp:
        s = "% d(%.2d)" % (_cint(rv), ev) if ee == 1 else "% .1f(%d.%d)x10^%d" % (mant, hi, lo, ee)
    elif ee - oexp == 1:
        m = abs(mant) if abs(mant) < 0.99999999999999 else mant
        s = "% .1f(%d.%d)x10^%d" % (m / 10.0, hi, lo, ee)
    elif ee > 1 and oexp > 1 and ee - oexp <= -1:
        s = "% .*f(%.2d)x10^%d" % (oexp - ee + 1, mant, ev, oexp)
    elif ee == 1 and oexp > 0:
        s = "% d(%.2d)" % (_cint(rv), ev)
    else:
        return None
    return _fin(s, length)


def _centre(s, width):
    if len(s) >= width:
        return s[:width]
    left = (width - len(s)) // 2
    return " " * left + s + " " * (width - left - len(s))


def _props(derivs, r, z, w):
    out = FourierProps()
    if _polish_lib().orc_calc_props(RDerivs(*[float(v) for v in derivs]), r, z, w,
                                    C.byref(out)):
        raise ValueError("calc_props: power or local power ~ 0")
    return out


def _rzwerrs(props, T):
    L = _polish_lib()
    L.orc_calc_rzwerrs.argtypes = [C.c_void_p, C.c_double, C.c_void_p]
    out = RzwErrs()
    if L.orc_calc_rzwerrs(C.addressof(props), T, C.addressof(out)):
        raise ValueError("calc_rzwerrs: T <= 0")
    return out


def _table_head(widths, t1, t2, skip):
    cols = [k for k in range(len(widths)) if k not in skip]
    lines = []
    for cells in ([_centre(t1[k], widths[k]) for k in cols],
                  [_centre(t2[k], widths[k]) for k in cols]):
        lines.append("  ".join(cells) + "\n")
    lines.append("--".join("-" * widths[k] for k in cols) + "\n")
    return "".join(lines)


def accelfile_text(T, nph, numw, cands, polished, inf_bytes=b""):
    """The reference's text candidate file for sorted, polished candidates
    ((power, sigma, numharm, r, z, w) and dicts of pows/hirs/hizs/hiws/derivs)
    of an observation of T seconds; nph > 0 for -photon; numw > 0 for a jerk
    search.  Returns bytes; notes are those of a telescope "None" run."""
    def ve(val, err, digits, width):
        s = nice_output_1(val, err) if digits == 1 else nice_output_2(val, err)
        if s is None:
            raise ValueError("nice_output_2: undefined condition")
        return _centre(s, width)

    sig = lib(64).orc_candidate_sigma
    sig.restype = C.c_double
    sig.argtypes = [C.c_double, C.c_int, C.c_double]
    f32 = np.float32
    props = []
    for c, p in zip(cands, polished):
        pr = _props(p["derivs"][0], c[3], c[4], c[5])
        pr.rerr = float(f32(0.5) / f32(c[2]))
        pr.zerr = float(f32(2.0) / f32(c[2]))
        pr.werr = float(f32(20.0) / f32(c[2]))
        props.append(pr)
    n = len(cands)
    notes = [" " * 20 for _ in range(n)]
    for i in range(n):
        for j in range(n):
            if i == j:
                continue
            if (abs(props[i].r - props[j].r) < 15.0 and abs(props[i].z - props[j].z) > 1.0
                    and props[i].pow > props[j].pow):
                if notes[j] == " " * 20:
                    notes[j] = ("SL? of Cand %d" % (i + 1))[:20]
                continue
            for k in range(1, 61):
                if (abs(props[i].r - props[j].r / k) < float(f32(props[j].rerr) * f32(3))
                        and abs(props[i].z - props[j].z / k) < float(f32(props[j].zerr) * f32(2))
                        and notes[j] == " " * 20):
                    notes[j] = ("H %d of Cand %d" % (k, i + 1))[:20]
                    break
    out = []
    fw = [4, 5, 6, 8, 4, 16, 15, 15, 15, 11, 11, 15, 20]
    out.append(_table_head(fw, ["", "", "Summed", "Coherent", "Num", "Period", "Frequency",
                                "FFT 'r'", "Freq Deriv", "FFT 'z'", "FFT 'w'", "Accel", ""],
                           ["Cand", "Sigma", "Power", "Power", "Harm", "(ms)", "(Hz)", "(bin)",
                            "(Hz/s)", "(bins)", "(bins)", "(m/s^2)", "Notes"],
                           () if numw else (10,)))
    for i, (c, p) in enumerate(zip(cands, polished)):
        er = _rzwerrs(props[i], T)
        phs0 = float(p["derivs"][0][1])
        cr = ci = 0.0
        for h in range(c[2]):
            d = [float(v) for v in p["derivs"][h]]
            amp = math.sqrt(d[0] / nph) if nph > 0.0 else math.sqrt(d[0] / d[6])
            corr = phs0 - math.fmod((h + 1.0) * phs0, 2.0 * math.pi)
            cr += amp * math.cos(d[1] + corr)
            ci += amp * math.sin(d[1] + corr)
        cells = [_centre("%-4d" % (i + 1), 4), _centre("%.2f" % c[1], 5),
                 _centre("%.2f" % c[0], 6), _centre("%.2f" % (cr * cr + ci * ci), 8),
                 _centre("%d" % c[2], 4), ve(er.p * 1000.0, er.perr * 1000.0, 1, 16),
                 ve(er.f, er.ferr, 1, 15), ve(props[i].r, props[i].rerr, 2, 15),
                 ve(er.fd, er.fderr, 1, 15), ve(props[i].z, props[i].zerr, 2, 11)]
        if numw:
            cells.append(ve(props[i].w, props[i].werr, 2, 11))
        cells.append(ve(props[i].z * SOL / (T * T * er.f), props[i].zerr * SOL / (T * T * er.f),
                        2, 15))
        out.append("  ".join(cells) + "    " + notes[i].split("\0")[0] + "\n")
    out.append("\n\n")
    hw = [5, 4, 5, 15, 11, 18, 13, 12, 9, 12, 9, 12, 10, 10, 20]
    out.append(_table_head(hw, ["", "", "", "Power /", "Raw", "FFT 'r'", "Pred 'r'", "FFT 'z'",
                                "Pred 'z'", "FFT 'w'", "Pred 'w'", "Phase", "Centroid", "Purity",
                                ""],
                           ["Cand", "Harm", "Sigma", "NumPhot" if nph > 0.0 else "Loc Pow",
                            "Power", "(bin)", "(bin)", "(bins)", "(bins)", "(bins)", "(bins)",
                            "(rad)", "(0-1)", "<p> = 1", "Notes"],
                           () if numw else (9, 10)))
    for i, (c, p) in enumerate(zip(cands, polished)):
        for h in range(c[2]):
            d = [float(v) for v in p["derivs"][h]]
            if nph > 0.0:
                d[6] = nph
            hp = _props(d, float(p["hirs"][h]), float(p["hizs"][h]), float(p["hiws"][h]))
            cells = [_centre(" %-4d" % (i + 1) if h == 0 else "     ", 5),
                     _centre("%-4d" % (h + 1), 4), _centre("%.2f" % sig(hp.pow, 1, 1.0), 5),
                     ve(hp.pow, hp.powerr, 2, 15), _centre("%.3g" % hp.rawpow, 11),
                     ve(hp.r, hp.rerr, 2, 18), _centre("%.2f" % (c[3] * (h + 1)), 13),
                     ve(hp.z, hp.zerr, 2, 12), _centre("%.2f" % (c[4] * (h + 1)), 9)]
            if numw:
                cells += [ve(hp.w, hp.werr, 2, 12), _centre("%.2f" % (c[5] * (h + 1)), 9)]
            cells += [ve(hp.phs, hp.phserr, 2, 12), ve(hp.cen, hp.cenerr, 2, 10),
                      ve(hp.pur, hp.purerr, 2, 10)]
            out.append("  ".join(cells) + "    " + " " * 20 + "\n")
    out.append("\n\n")
    return "".join(out).encode() + inf_bytes


def ref_dedisp_lib():
    """oracle/_ref/libref_dedisp.so (src/dispersion.c compiled unmodified), or
    None where the reference tree was not at hand."""
    path = os.path.join(HERE, "_ref", "libref_dedisp.so")
    if not os.path.exists(path):
        return None
    if path not in _libs:
        L = C.CDLL(path)
        dp = C.POINTER(C.c_double)
        for name in ("dedisp_delays", "subband_delays"):
            getattr(L, name).restype = dp
        L.dedisp_delays.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double]
        L.subband_delays.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                     C.c_double]
        L.subband_search_delays.restype = dp
        L.subband_search_delays.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                            C.c_double]
        L.dedisp_subbands.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                      C.c_int, C.c_void_p]
        L.float_dedisp.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                   C.c_float, C.c_void_p]
        L.vect_free.argtypes = [C.c_void_p]
        _libs[path] = L
    return _libs[path]


def _nearest_long(x):
    return int(np.ceil(x - 0.5)) if x < 0 else int(np.floor(x + 0.5))


def ref_dedisp_delays(L, nchan, lofreq, chanwidth, dt, nsub, dms, ds):
    """prepsubband's integer delays (src/prepsubband.c:365-390) from the
    reference's own subband_search_delays / subband_delays."""
    avgdm = 0.0
    for d in dms:
        avgdm += d
    avgdm /= len(dms)
    p = L.subband_search_delays(nchan, nsub, avgdm, lofreq, chanwidth, 0.0)
    cd = np.array([_nearest_long(p[i] / dt) for i in range(nchan)], np.int32)
    L.vect_free(p)
    off = np.zeros((len(dms), nsub), np.int32)
    for i, dm in enumerate(dms):
        q = L.subband_delays(nchan, nsub, float(dm), lofreq, chanwidth, 0.0)
        top = q[nsub - 1]
        off[i] = [_nearest_long((q[j] - top) / (dt * ds)) for j in range(nsub)]
        L.vect_free(q)
    return cd, off


def ref_dedisperse(L, X, lofreq, chanwidth, dt, nsub, dms, ds, W):
    """prepsubband's dedispersion over the reference's own dedisp_subbands
    and float_dedisp, streamed in blocks of W spectra as the program streams
    them (src/backend_common.c:660-758 prep_subbands; src/prepsubband.c:
    919-1025 get_data): each stage pairs a block with the next (lastdata,
    data), the raw blocks transposed to channel-major, the subband blocks
    back to time-major, downsampled by averaging (float sums, then / ds), the
    data followed by zero blocks.  X: time-major float32 [nspec][nchan],
    nspec a multiple of W, W of ds.  Returns out[ndm][nspec // ds]."""
    nspec, nchan = X.shape
    nb = nspec // W
    cd, off = ref_dedisp_delays(L, nchan, lofreq, chanwidth, dt, nsub, dms, ds)
    zeros = np.zeros((W, nchan), np.float32)
    raw = [np.ascontiguousarray(X[b * W:(b + 1) * W].T) for b in range(nb)] + \
        [np.ascontiguousarray(zeros.T)] * 2
    sub = []                                    # time-major [W][nsub] per block
    for b in range(nb + 1):
        res = np.zeros(nsub * W, np.float32)
        L.dedisp_subbands(raw[b + 1].ctypes.data, raw[b].ctypes.data, W, nchan, cd.ctypes.data,
                          nsub, res.ctypes.data)
        s = res.reshape(nsub, W).T.copy()
        if ds > 1:
            ftmp = np.zeros((W // ds, nsub), np.float32)
            for k in range(ds):
                ftmp = (ftmp + s[k::ds]).astype(np.float32)
            s = (np.float32(0.0) + ftmp / np.float32(ds)).astype(np.float32)
        sub.append(np.ascontiguousarray(s))
    n = W // ds
    out = np.zeros((len(dms), nb * n), np.float32)
    res = np.zeros(n, np.float32)
    for b in range(nb):
        for i in range(len(dms)):
            o = np.ascontiguousarray(off[i])
            L.float_dedisp(sub[b + 1].ctypes.data, sub[b].ctypes.data, n, nsub, o.ctypes.data,
                           0.0, res.ctypes.data)
            out[i, b * n:(b + 1) * n] = res
    return out
