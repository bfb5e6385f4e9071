"""Learned Sommerfeld surrogate: an MLP that predicts the remainder surfaces.

The reference evaluates the Sommerfeld remainder by interpolating four
surfaces (I_rho^V, I_z^V, I_rho^H, I_phi^H) from a grid it fills by contour
quadrature for every (eps, r1) bucket (``_sommerfeld.py:648-1116``).  This
module replaces the grid with a small network trained once on values of the
project's own quadrature (``mw_somm_surfaces_eps``):

    inputs   (rho, z+z') as the normalised polar pair (R1/lambda, theta),
             log|eps~|, arg eps~, log f                        (5 features)
    network  4 hidden layers of width 128, GELU, BF16 weights, FP32 accumulation
    outputs  Re/Im of the four surfaces at the wavelength-normalised master
             scale (k2 = 2 pi, omega = 2 pi c, mu = 4e-7 pi), divided by SCALE

Physical surfaces are the outputs x SCALE x (omega mu) / (omega0 mu0), the
same frequency factor a scaled grid carries.  The forward, backward and Adam
steps are hand-written CUDA (``mlp.cu``); inference runs on tcgen05 tensor
cores, standalone (``mw_mlp_infer``) or fused into the remainder fill
(``mw_somm_remainder_q_mlp``).  Queries outside ``DOMAIN`` and structures
whose spot check against quadrature misses the error tolerance take the
grid path instead.

Accuracy.  The shipped network reproduces the surfaces to about 1e-3 of
their size (held-out rms 2.5e-3 of SCALE), which moves drive-point
impedances by 1e-4 to 3e-3 -- far outside the 1e-6 that the mixed-precision
path holds to.  A structure is therefore served only when the spot check's
relative surface error is within the solver's ``surrogate_tol``: at the
default, ``DEFAULT_TOL`` = 1e-6, the shipped network serves no structure of
the seeded Sommerfeld workload and every solve takes the quadrature grid;
with ``surrogate_tol=APPROX_TOL`` it serves them as an approximation, which
is not counted toward the 1e-6 gate.
"""

from __future__ import annotations

import math
import time
from pathlib import Path

import numpy as np

from . import _lib

C_LIGHT = 299_792_458.0
EPS0 = 8.8541878188e-12
MU0_GRID = 4e-7 * math.pi
K2_REF = 2.0 * math.pi
OMEGA_REF = K2_REF * C_LIGHT
SCALE = 200.0

# training / validity domain
R1_MAX_WL = 4.0
H_MIN_WL = 0.02
EPS_ABS = (2.0, 1000.0)
F_HZ = (2.5e6, 35e6)

WEIGHTS_PATH = Path(__file__).resolve().parent / "data" / "somm_mlp.npz"

# spot check: node pairs sampled per structure; the surrogate serves a
# structure when max |surrogate - quadrature| / max |quadrature| over them
# is within the solver's surrogate_tol
SPOT_PAIRS = 64
DEFAULT_TOL = 1e-6
# the approximation setting: the shipped network serves the seeded
# structures at drive-point impedances within ZIN_TOL of the grid path
APPROX_TOL = 2e-2
ZIN_TOL = 1e-2


def _torch():
    import torch

    return torch


def features(rho_wl, h_wl, eps, f_hz):
    """(n, 5) float32 network inputs from rho and z+z' in wavelengths, the
    complex relative permittivity eps~ and the frequency."""
    rho = np.asarray(rho_wl, dtype=np.float64)
    h = np.asarray(h_wl, dtype=np.float64)
    rho, h, eps, f = np.broadcast_arrays(rho, h, np.asarray(eps, dtype=np.complex128),
                                         np.asarray(f_hz, dtype=np.float64))
    r1 = np.hypot(rho, h)
    th = np.arctan2(h, rho)
    x = np.empty(rho.shape + (5,), dtype=np.float64)
    x[..., 0] = 2.0 * np.sqrt(np.minimum(r1, R1_MAX_WL) / R1_MAX_WL) - 1.0
    x[..., 1] = 4.0 * th / math.pi - 1.0
    la, lo, hi = np.log(np.abs(eps)), math.log(EPS_ABS[0]), math.log(EPS_ABS[1])
    x[..., 2] = 2.0 * (la - lo) / (hi - lo) - 1.0
    x[..., 3] = 2.0 * np.angle(eps) / (-0.5 * math.pi) - 1.0
    lf, flo, fhi = np.log(f), math.log(F_HZ[0]), math.log(F_HZ[1])
    x[..., 4] = 2.0 * (lf - flo) / (fhi - flo) - 1.0
    return x.astype(np.float32)


def in_domain(rho_wl, h_wl, eps, f_hz):
    """Boolean mask of queries inside the training domain."""
    rho = np.asarray(rho_wl, dtype=np.float64)
    h = np.asarray(h_wl, dtype=np.float64)
    eps = np.asarray(eps, dtype=np.complex128)
    f = np.asarray(f_hz, dtype=np.float64)
    a = np.abs(eps)
    return ((np.hypot(rho, h) <= R1_MAX_WL) & (h >= H_MIN_WL) & (a >= EPS_ABS[0]) & (a <= EPS_ABS[1])
            & (eps.imag <= 0.0) & (f >= F_HZ[0]) & (f <= F_HZ[1]))


def sample_domain(n, rng):
    """Training queries: z+z' log-uniform, rho half uniform and half
    log-uniform, eps~ from eps_r U(2.5, 45) and sigma log-U(5e-5, 0.2) S/m,
    f log-U over the frequency range; R1 <= R1_MAX_WL."""
    h = np.exp(rng.uniform(math.log(H_MIN_WL), math.log(R1_MAX_WL), n))
    rho = np.where(rng.random(n) < 0.5, rng.uniform(0.0, R1_MAX_WL, n),
                   np.exp(rng.uniform(math.log(1e-3), math.log(R1_MAX_WL), n)))
    r1 = np.hypot(rho, h)
    s = np.where(r1 > R1_MAX_WL, R1_MAX_WL / r1 * rng.uniform(0.3, 1.0, n), 1.0)
    rho, h = rho * s, np.maximum(h * s, H_MIN_WL)
    er = rng.uniform(2.5, 45.0, n)
    sig = np.exp(rng.uniform(math.log(5e-5), math.log(0.2), n))
    f = np.exp(rng.uniform(math.log(F_HZ[0]), math.log(F_HZ[1]), n))
    eps = er - 1j * sig / (2.0 * math.pi * f * EPS0)
    bad = np.abs(eps) > EPS_ABS[1]
    eps[bad] = eps[bad] / np.abs(eps[bad]) * EPS_ABS[1] * 0.999
    return rho, h, eps, f


def quadrature_surfaces(rho_wl, h_wl, eps, device, stream=None, rtol=1e-6):
    """(n, 4) complex128 surfaces at the master normalisation by the six
    contour integrals (``mw_somm_surfaces_eps``); a device tensor."""
    torch = _torch()
    rho = np.asarray(rho_wl, dtype=np.float64)
    h = np.asarray(h_wl, dtype=np.float64)
    eps = np.asarray(eps, dtype=np.complex128)
    r1 = np.hypot(rho, h)
    th = np.arctan2(h, rho)
    host = np.ascontiguousarray(np.stack([r1, rho, h, th, eps.real, eps.imag]))
    d = torch.from_numpy(host).to(device)
    out = torch.empty((rho.size, 4), dtype=torch.complex128, device=device)
    ws = torch.empty(256, dtype=torch.uint8, device=device)
    st = stream if stream is not None else torch.cuda.current_stream(device).cuda_stream
    _lib.call("mw_somm_surfaces_eps", rho.size, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
              d[3].data_ptr(), d[4].data_ptr(), d[5].data_ptr(), K2_REF, OMEGA_REF, MU0_GRID, float(rtol),
              out.data_ptr(), ws.data_ptr(), st)
    return out


def targets_from_surfaces(s):
    """(n, 8) float32 targets (Re/Im of the 4 surfaces / SCALE)."""
    torch = _torch()
    return (torch.view_as_real(s).reshape(s.shape[0], 8) / SCALE).float()


class Surrogate:
    """Network parameters resident on one device (FP32 master + BF16)."""

    def __init__(self, params, device):
        torch = _torch()
        lib = _lib.load()
        n = int(lib.mw_mlp_param_count())
        params = np.asarray(params, dtype=np.float32).ravel()
        if params.size != n:
            raise ValueError(f"expected {n} parameters, got {params.size}")
        self.device = device
        self.p32 = torch.from_numpy(params.copy()).to(device)
        self.pbf = torch.empty(n, dtype=torch.int16, device=device)  # BF16 bits
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        _lib.call("mw_mlp_to_bf16", self.p32.data_ptr(), self.pbf.data_ptr(), self._stream())
        self.meta = {}

    def _stream(self):
        return _torch().cuda.current_stream(self.device).cuda_stream

    @classmethod
    def load(cls, device, path=WEIGHTS_PATH):
        d = np.load(path)
        s = cls(d["params"], device)
        s.meta = {k: d[k] for k in d.files if k != "params"}
        return s

    def save(self, path=WEIGHTS_PATH, **meta):
        Path(path).parent.mkdir(parents=True, exist_ok=True)
        np.savez(path, params=self.p32.cpu().numpy(), **meta)

    def predict(self, X):
        """(n, 8) float32 outputs for (n, 5) features (tensor-core path)."""
        torch = _torch()
        X = torch.as_tensor(X, dtype=torch.float32, device=self.device).contiguous()
        Y = torch.empty((X.shape[0], 8), dtype=torch.float32, device=self.device)
        _lib.call("mw_mlp_infer", X.shape[0], X.data_ptr(), self.pbf.data_ptr(), self.p32.data_ptr(), Y.data_ptr(),
                  self.err.data_ptr(), self._stream())
        return Y

    def predict_fp32(self, X):
        """(n, 8) outputs of the FP32 training forward (SIMT kernels)."""
        torch = _torch()
        X = torch.as_tensor(X, dtype=torch.float32, device=self.device).contiguous()
        n = X.shape[0]
        Y = torch.empty((n, 8), dtype=torch.float32, device=self.device)
        wsb = _lib.load().mw_mlp_train_workspace_size(n)
        ws = torch.empty(wsb, dtype=torch.uint8, device=self.device)
        _lib.call("mw_mlp_forward", n, X.data_ptr(), self.pbf.data_ptr(), self.p32.data_ptr(), Y.data_ptr(),
                  ws.data_ptr(), wsb, self._stream())
        return Y

    def surfaces(self, rho_wl, h_wl, eps, f_hz):
        """(n, 4) complex128 surfaces at the master normalisation."""
        torch = _torch()
        Y = self.predict(features(rho_wl, h_wl, eps, f_hz)).double() * SCALE
        return torch.view_as_complex(Y.reshape(-1, 4, 2).contiguous())


def generate(n, seed, device, chunk=1 << 20):
    """n training rows: (X (n, 5) float32, T (n, 8) float32) device tensors."""
    torch = _torch()
    rng = np.random.default_rng(seed)
    Xs, Ts = [], []
    for c0 in range(0, n, chunk):
        m = min(chunk, n - c0)
        rho, h, eps, f = sample_domain(m, rng)
        Xs.append(torch.from_numpy(features(rho, h, eps, f)).to(device))
        Ts.append(targets_from_surfaces(quadrature_surfaces(rho, h, eps, device)))
    return torch.cat(Xs), torch.cat(Ts)


def train(n_samples=10_000_000, epochs=30, batch=8192, lr=2e-3, lr_min=2e-5, seed=0, device=None, data=None,
          log=print):
    """Train a surrogate from scratch on quadrature data with Adam and a
    cosine learning-rate decay.  Returns (Surrogate, history), history a list
    of (epoch, mean batch loss, seconds)."""
    torch = _torch()
    device = device or torch.device("cuda", 0)
    t0 = time.perf_counter()
    X, T = data if data is not None else generate(n_samples, seed, device)
    torch.cuda.synchronize(device)
    log(f"data: {X.shape[0]} rows in {time.perf_counter() - t0:.1f} s")
    model = Surrogate(he_init(seed), device)
    lib = _lib.load()
    n_par = int(lib.mw_mlp_param_count())
    m = torch.zeros(n_par, dtype=torch.float32, device=device)
    v = torch.zeros(n_par, dtype=torch.float32, device=device)
    loss = torch.zeros(1, dtype=torch.float32, device=device)
    wsb = lib.mw_mlp_train_workspace_size(batch)
    ws = torch.empty(wsb, dtype=torch.uint8, device=device)
    st = torch.cuda.current_stream(device).cuda_stream
    n = X.shape[0]
    steps_per_epoch = n // batch
    total = steps_per_epoch * epochs
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    history, step = [], 0
    for ep in range(epochs):
        perm = torch.randperm(n, device=device, generator=gen)
        loss.zero_()
        for b in range(steps_per_epoch):
            rows = perm[b * batch:(b + 1) * batch]
            step += 1
            lr_t = lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * step / total))
            _lib.call("mw_mlp_train_step", batch, X.data_ptr(), T.data_ptr(), rows.data_ptr(), model.p32.data_ptr(),
                      model.pbf.data_ptr(), m.data_ptr(), v.data_ptr(), step, lr_t, 0.9, 0.999, 1e-8,
                      loss.data_ptr(), ws.data_ptr(), wsb, st)
        mean = float(loss.item()) / max(steps_per_epoch, 1)
        history.append((ep, mean, time.perf_counter() - t0))
        log(f"epoch {ep}: loss {mean:.3e} ({time.perf_counter() - t0:.1f} s)")
    return model, history


def evaluate(model, rho_wl, h_wl, eps, f_hz):
    """Errors of the tensor-core surrogate against quadrature on the given
    queries: (max |dS| / SCALE, rms |dS| / SCALE, per-query max error)."""
    torch = _torch()
    q = quadrature_surfaces(rho_wl, h_wl, eps, model.device)
    p = model.surfaces(rho_wl, h_wl, eps, f_hz)
    e = (p - q).abs().max(dim=1).values / SCALE
    return float(e.max()), float(torch.sqrt((e * e).mean())), e


def he_init(seed):
    """He-normal weights, zero biases, flat layout [W_l (out x in), b_l]."""
    rng = np.random.default_rng(seed)
    dims = [(5, 128), (128, 128), (128, 128), (128, 128), (128, 8)]
    parts = []
    for i, n in dims:
        parts.append((rng.standard_normal(i * n) * math.sqrt(2.0 / i)).astype(np.float32))
        parts.append(np.zeros(n, dtype=np.float32))
    return np.concatenate(parts)


_MODELS: dict = {}


def get_model(device):
    """The shipped surrogate on `device` (loaded once), or None without
    weights."""
    key = getattr(device, "index", None)
    if key not in _MODELS:
        _MODELS[key] = Surrogate.load(device) if WEIGHTS_PATH.exists() else None
    return _MODELS[key]


def spot_check(model, rho_wl, h_wl, eps, f_hz):
    """(largest |surrogate - quadrature| / SCALE, the same relative to the
    largest |quadrature|) over the given queries."""
    q = quadrature_surfaces(rho_wl, h_wl, np.full(np.shape(rho_wl), eps), model.device)
    p = model.surfaces(rho_wl, h_wl, eps, f_hz)
    d = float((p - q).abs().max())
    return d / SCALE, d / max(float(q.abs().max()), 1e-300)
