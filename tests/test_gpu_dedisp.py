"""Subband dedispersion on the device (ab_dedisperse) against the reference's
own dedisp_subbands / float_dedisp streamed as prepsubband streams them
(oracle/_ref/libref_dedisp.so), bit for bit, from host and from device
memory; and the DM trial it produces carries an injected dispersed pulsar
into the search at its DM."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
LO, BW, DT = 1200.0, 1.0, 1e-4


def _spectra(nspec, nchan, seed, dm=None, f0=None):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((nspec, nchan)).astype(np.float32)
    if dm is not None:
        # a pulse train at f0 Hz, delayed per channel by the cold-plasma delay
        t = np.arange(nspec) * DT
        freqs = LO + BW * np.arange(nchan)
        delay = dm / (0.000241 * freqs ** 2)
        delay -= delay[-1]
        for c in range(nchan):
            ph = (t - delay[c]) * f0
            X[:, c] += (1.5 * (np.cos(2 * np.pi * ph) > 0.95)).astype(np.float32)
    return X


@pytest.mark.parametrize("nchan,nsub,ds,dmstep", [(64, 8, 1, 5.0), (64, 16, 2, 5.0),
                                                  (128, 8, 4, 5.0), (128, 16, 1, 23.0),
                                                  (32, 32, 3, 61.0), (256, 8, 1, 11.0),
                                                  (96, 8, 2, 7.0), (128, 2, 1, 10.0),
                                                  (64, 32, 2, 13.0)])
def test_dedisperse_matches_streamed_reference(ctx, oracle, nchan, nsub, ds, dmstep):
    """1, 2, 4, 8, 16, 32 and 64 channels per subband (the compiled widths)
    and 12 (the general path); DM steps of 23, 61, 11 and 13 (14, 4, 28 and 24
    trials: ragged last groups of 16 DMs, a group of 8, wide offset spreads
    within a group); an odd downsampling factor among the cases."""
    L = oracle.ref_dedisp_lib()
    if L is None:
        pytest.skip("oracle/_ref/libref_dedisp.so is built where the reference tree is present")
    W, nb = 4096 - 4096 % ds, 4                   # blocks of a multiple of ds spectra
    X = _spectra(W * nb, nchan, nchan + ds, dm=60.0, f0=37.0)
    dms = np.arange(0.0, 200.0 if dmstep < 10 else 300.0, dmstep)
    want = oracle.ref_dedisperse(L, X, LO, BW, DT, nsub, dms, ds, W)
    got = ctx.dedisperse(X, LO, BW, DT, nsub, dms, downsamp=ds)
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_dedisperse_device_buffers(ctx):
    import torch

    X = _spectra(1 << 14, 64, 3)
    dms = np.arange(0.0, 100.0, 10.0)
    host = ctx.dedisperse(X, LO, BW, DT, 8, dms)
    dx = torch.from_numpy(X).cuda()
    dout = torch.empty((dms.size, X.shape[0]), dtype=torch.float32, device="cuda")
    ctx.dedisperse(None, LO, BW, DT, 8, dms, device_ptr=dx.data_ptr(), nspec=X.shape[0],
                   nchan=X.shape[1], out_ptr=dout.data_ptr())
    assert np.array_equal(dout.cpu().numpy().view(np.uint32), host.view(np.uint32))


def test_dedispersed_trial_finds_the_pulsar(ctx, ablib):
    """N = 2^17 samples of 64 channels with a pulsar at DM 60, f = 37 Hz: the
    DM-60 trial's strongest candidate is the pulsar; the DM-0 trial's signal
    is smeared far below it."""
    N = 1 << 17
    X = _spectra(N, 64, 11, dm=60.0, f0=37.0)
    trials = ctx.dedisperse(X, LO, BW, DT, 8, [0.0, 60.0])
    s = ablib.AccelSearch(zmax=10, numharm=8, sigma=2.0, ctx=ctx)
    best = {}
    for i, dm in enumerate((0.0, 60.0)):
        fft = ctx.series_to_fft(trials[i], DT)
        cands = s(fft, N, DT)
        best[dm] = max(cands, key=lambda c: c[1]) if cands else None
    T = N * DT
    top = best[60.0]
    assert top is not None
    # the candidate is the pulsar or a harmonic relative of it
    ratio = top[3] / (37.0 * T)
    assert min(abs(ratio - p / q) for p in range(1, 9) for q in range(1, 9)) < 0.01, top
    assert best[0.0] is None or best[0.0][1] < top[1]


@pytest.mark.parametrize("nspec,ds", [(1 << 16, 1), ((1 << 16) + 2, 2)])
def test_search_dedispersed_equals_host_chain(ctx, ablib, nspec, ds):
    """ab_search_dedispersed (trials and their spectra stay on the device)
    gives, trial by trial, exactly the candidates of the same steps chained
    through host arrays: ab_dedisperse, ab_series_to_fft, ab_search.  With
    ds = 2 the trials have an odd length and lose their last sample; the
    pulsar at DM 60 is the strongest candidate of its trial."""
    X = _spectra(nspec, 64, 21, dm=60.0, f0=37.0)
    dms = [0.0, 30.0, 60.0, 90.0]
    n = (nspec // ds) & ~1
    obs = ablib.obs_init(ablib.make_params(n, DT * ds, n // 2, zmax=10, numharm=4, sigma=2.0))
    got = ctx.search_dedispersed(X, LO, BW, DT, 8, dms, obs, downsamp=ds)
    trials = ctx.dedisperse(X, LO, BW, DT, 8, dms, downsamp=ds)
    assert len(got) == len(dms)
    for d in range(len(dms)):
        fft = ctx.series_to_fft(trials[d][:n], DT * ds)
        want = ctx.search(obs, fft)
        assert got[d] == want, d
    top = max(got[2], key=lambda c: c[1])
    ratio = top[3] / (37.0 * n * DT * ds)
    assert min(abs(ratio - p / q) for p in range(1, 9) for q in range(1, 9)) < 0.01, top


def test_search_dedispersed_device_input_and_checks(ctx, ablib):
    """Spectra already on the device give the host input's result; an obs that
    does not describe the trials is refused."""
    import torch

    X = _spectra(1 << 15, 32, 5, dm=40.0, f0=29.0)
    dms = [0.0, 40.0]
    n = X.shape[0]
    obs = ablib.obs_init(ablib.make_params(n, DT, n // 2, zmax=6, numharm=2, sigma=2.0))
    host = ctx.search_dedispersed(X, LO, BW, DT, 4, dms, obs)
    dx = torch.from_numpy(X).cuda()
    dev = ctx.search_dedispersed(None, LO, BW, DT, 4, dms, obs, device_ptr=dx.data_ptr(),
                                 nspec=X.shape[0], nchan=X.shape[1])
    assert dev == host and sum(len(c) for c in host) > 0
    bad = ablib.obs_init(ablib.make_params(n // 2, DT, n // 4, zmax=6, numharm=2, sigma=2.0))
    with pytest.raises(ablib.AccelError):
        ctx.search_dedispersed(X, LO, BW, DT, 4, dms, bad)


def test_dedisperse_large_host_input_equals_device_input(ctx):
    """A 512 MB host array (1024 channels x 2^17 spectra) goes up through the
    pinned, multi-threaded staging; the trials equal those of the same spectra
    handed over in device memory, bit for bit, on two calls in a row."""
    import torch

    rng = np.random.default_rng(31)
    X = rng.standard_normal((1 << 17, 1024), dtype=np.float32)
    dms = np.linspace(0.0, 300.0, 24)
    host = ctx.dedisperse(X, 1400.0, 0.25, 64e-6, 64, dms)
    dx = torch.from_numpy(X).cuda()
    dout = torch.empty((dms.size, X.shape[0]), dtype=torch.float32, device="cuda")
    ctx.dedisperse(None, 1400.0, 0.25, 64e-6, 64, dms, device_ptr=dx.data_ptr(),
                   nspec=X.shape[0], nchan=X.shape[1], out_ptr=dout.data_ptr())
    assert np.array_equal(dout.cpu().numpy().view(np.uint32), host.view(np.uint32))
    again = ctx.dedisperse(X, 1400.0, 0.25, 64e-6, 64, dms)   # staging buffers reused
    assert np.array_equal(again.view(np.uint32), host.view(np.uint32))
