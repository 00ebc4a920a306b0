"""Learned warm start for CW sweeps.

An MLP maps an instance's sweep parameters (pump ratio N, detuning delta,
intracavity GDD, reflectivity R) to a description of its steady-state
signal; the batched solver then starts that instance from the predicted
field instead of noise.  Two output representations (512 values each):

* "low_modes": the 256 lowest Fourier modes (complex) of the steady state;
* "band": the steady state of these detuned, dispersive cavities is a
  signal/idler pair of bands around +-q0 (measured: >= 98 % of the power
  within +-64 modes of the strongest pair for 90 % of the converged
  instances, q0 up to ~3000 of 4096, reproducible between noise seeds to a
  few modes), and the phase Phi of every pair product c_q c_-q is set by the
  pump (coherent across the band to 0.998 and between seeds to 0.015 rad),
  while the relative phases inside a band are not reproducible.  So the
  network predicts the 2 x 128 band magnitudes, Phi, q0 and the power, and
  the field is synthesised with every pair at phase Phi.  The network is the library's tensor-core
MLP (cuopo_mlp_*, BF16 on tcgen05 with FP32 accumulation); the fields are
made and read with the library's own FFT (cuopo_fft_c2c) and the
spectrum/mode kernels.  A prediction is used only if it passes a one-round-
trip check (relative change of the signal power below `check_tol`) and
predicts a power above `p_min`; every other instance starts from the same
seeded noise as a plain solve.  The reference has no counterpart (it starts
every run from noise, src/headers/functions.cuh:58-71).
"""
from __future__ import annotations

import ast
import ctypes as C
import time
from pathlib import Path

import numpy as np

from . import api
from ._lib import check, load

N_MODES = 256
N_FEATURES = 4
BAND = 128          # modes per band of the band representation
MAG_SCALE = 8.0     # band magnitudes are stored with unit norm x MAG_SCALE
WIDTH = 512
DEPTH = 4
# feature normalisation of the sweep's ranges to [-1, 1]
FEAT_CENTER = np.array([3.6, 0.0, 0.0, 0.945])
FEAT_HALF = np.array([2.4, np.pi, 500.0, 0.045])
DATA_DIR = Path(__file__).resolve().parent / "data"
MODEL_PATH = DATA_DIR / "warmstart_mlp.npz"


def _torch():
    import torch
    return torch


def _stream(stream):
    torch = _torch()
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


class MLP:
    """The library's tensor-core MLP (cuopo_mlp_*): n_in -> width (GELU) x depth -> n_out."""

    def __init__(self, n_in: int = N_FEATURES, width: int = WIDTH, depth: int = DEPTH, n_out: int = 2 * N_MODES,
                 max_batch: int = 4096, seed: int = 0):
        self._lib = load()
        h = C.c_void_p()
        check(self._lib.cuopo_mlp_create(C.byref(h), n_in, width, depth, n_out, max_batch, seed))
        self._h = h
        self.n_in, self.width, self.depth, self.n_out, self.max_batch = n_in, width, depth, n_out, max_batch
        n = C.c_long()
        check(self._lib.cuopo_mlp_param_count(self._h, C.byref(n)))
        self.n_params = n.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.cuopo_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        check(self._lib.cuopo_mlp_get_params(self._h, out.ctypes.data))
        return out

    def set_params(self, params) -> None:
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == self.n_params
        check(self._lib.cuopo_mlp_set_params(self._h, p.ctypes.data))

    def forward(self, x, stream=None):
        """x: CUDA float32 [B][n_in] -> CUDA float32 [B][n_out] (chunks of max_batch)."""
        torch = _torch()
        x = x.contiguous().float()
        y = torch.empty(x.shape[0], self.n_out, dtype=torch.float32, device=x.device)
        for s in range(0, x.shape[0], self.max_batch):
            e = min(x.shape[0], s + self.max_batch)
            check(self._lib.cuopo_mlp_forward(self._h, x[s:e].data_ptr(), y[s:e].data_ptr(), e - s, _stream(stream)))
        return y

    def gradients(self, x, t, stream=None):
        """Loss and flat gradient (numpy float32) of the batch, without an update."""
        x = x.contiguous().float()
        t = t.contiguous().float()
        g = np.zeros(self.n_params, np.float32)
        loss = C.c_float()
        check(self._lib.cuopo_mlp_gradients(self._h, x.data_ptr(), t.data_ptr(), x.shape[0], g.ctypes.data,
                                            C.byref(loss), _stream(stream)))
        return float(loss.value), g

    def train_step(self, x, t, lr: float, loss=None, stream=None) -> None:
        """One Adam step (asynchronous; loss: CUDA float32 scalar tensor or None)."""
        check(self._lib.cuopo_mlp_train_step(self._h, x.data_ptr(), t.data_ptr(), x.shape[0], float(lr),
                                             None if loss is None else loss.data_ptr(), _stream(stream)))

    def status(self) -> None:
        check(self._lib.cuopo_mlp_status(self._h))

    def grad_step(self, x, t, loss=None, stream=None) -> None:
        """Forward, loss and backward on the batch into the network's gradient buffer (asynchronous)."""
        check(self._lib.cuopo_mlp_grad_step(self._h, x.data_ptr(), t.data_ptr(), x.shape[0],
                                            None if loss is None else loss.data_ptr(), _stream(stream)))

    def grad_tensor(self):
        """The network's device gradient buffer as a CUDA float32 tensor (a view, no copy)."""
        torch = _torch()
        ptr = C.POINTER(C.c_float)()
        n = C.c_long()
        check(self._lib.cuopo_mlp_grad_buffer(self._h, C.byref(ptr), C.byref(n)))

        class _View:
            __cuda_array_interface__ = {"shape": (n.value,), "typestr": "<f4",
                                        "data": (C.cast(ptr, C.c_void_p).value, False), "version": 2}
        return torch.as_tensor(_View(), device="cuda")

    def apply_adam(self, lr: float, grad_scale: float = 1.0, stream=None) -> None:
        """One Adam step from the gradient buffer times grad_scale (asynchronous)."""
        check(self._lib.cuopo_mlp_apply_adam(self._h, float(lr), float(grad_scale), _stream(stream)))


def gemm_bf16(A, B, split: int = 1, err=None, flags: int = 0, out=None, stream=None):
    """C = A B^T on the tensor cores (A [M][K], B [N][K] CUDA bfloat16) -> float32 [M][N]."""
    torch = _torch()
    M, K = A.shape
    N = B.shape[0]
    Cm = torch.empty(M, N, dtype=torch.float32, device=A.device) if out is None else out
    check(load().cuopo_gemm_bf16(A.data_ptr(), B.data_ptr(), Cm.data_ptr(), M, N, K, split, flags,
                                 None if err is None else err.data_ptr(), _stream(stream)))
    return Cm


# ------------------------------------------------------------ fields <-> modes

def modes_to_fields(modes, n_t: int, scale: float = 1.0, stream=None):
    """modes: CUDA float32 [count][2 N_MODES] -> time-domain fields, CUDA complex64 [count][n_t]."""
    torch = _torch()
    count = modes.shape[0]
    out = torch.empty(count, n_t, dtype=torch.complex64, device=modes.device)
    check(load().cuopo_fields_from_modes(modes.contiguous().data_ptr(), count, modes.shape[1] // 2, n_t, scale,
                                         out.data_ptr(), _stream(stream)))
    return out


def fields_to_modes(fields, n_t: int, scale: float = 1.0, n_modes: int = N_MODES, stream=None):
    """fields: CUDA complex64 [count][n_t] -> modes float32 [count][2 n_modes] (canonical sign)."""
    torch = _torch()
    fields = fields.reshape(-1, n_t).contiguous()
    count = fields.shape[0]
    spec = torch.empty_like(fields)
    api.fft_c2c(fields, -1, out=spec, stream=stream)
    modes = torch.empty(count, 2 * n_modes, dtype=torch.float32, device=fields.device)
    check(load().cuopo_modes_from_spectrum(spec.data_ptr(), count, n_t, n_modes, scale, modes.data_ptr(),
                                           _stream(stream)))
    return modes


def centre_code(q0, n_t: int):
    """The band centre as the network predicts it: 2 (q0 / (n_t/2))^2 - 1
    (q0^2 is close to linear in the cavity detuning; the synthesis kernel
    inverts it)."""
    return 2.0 * (q0 / (n_t / 2)) ** 2 - 1.0


def centre_decode(code, n_t: int):
    return np.clip(np.rint(np.sqrt(np.maximum(0.5 * (np.asarray(code) + 1.0), 0.0)) * (n_t / 2)),
                   BAND // 2, n_t // 2 - BAND // 2)


def band_targets(fields, ps, n_t: int, stream=None):
    """Training targets of the band representation from converged fields
    (CUDA complex64 [count][n_t]) and their signal powers: the library's FFT
    gives the modes c_q; the strongest signal/idler pair |c_q|^2 + |c_-q|^2
    sets q0; rows as cuopo_fields_from_bands reads them."""
    torch = _torch()
    fields = fields.reshape(-1, n_t).contiguous()
    count = fields.shape[0]
    X = torch.empty_like(fields)
    api.fft_c2c(fields, -1, out=X, stream=stream)
    c = X / n_t
    P = c.real ** 2 + c.imag ** 2
    q = torch.arange(1, n_t // 2, device=fields.device)
    pair = P[:, q] + P[:, (n_t - q) % n_t]
    q0 = q[torch.argmax(pair, dim=1)].clamp(BAND // 2, n_t // 2 - BAND // 2)
    k = torch.arange(BAND, device=fields.device)
    ip = (q0[:, None] - BAND // 2 + k[None, :]) % n_t
    im = (-q0[:, None] - BAND // 2 + k[None, :]) % n_t
    cp = torch.gather(c, 1, ip)
    cm = torch.gather(c, 1, im)
    mags = torch.cat([cp.abs(), cm.abs()], dim=1)
    mags = MAG_SCALE * mags / mags.norm(dim=1, keepdim=True).clamp_min(1e-30)
    # pair k of the + band (q = q0-64+k) is mode 128-k of the - band
    prod = (cp[:, 1:] * cm.flip(1)[:, :BAND - 1]).sum(dim=1)
    phi = torch.angle(prod)
    y = torch.empty(count, 512, dtype=torch.float32, device=fields.device)
    y[:, :2 * BAND] = mags
    y[:, 256:320] = torch.cos(phi)[:, None]
    y[:, 320:384] = torch.sin(phi)[:, None]
    y[:, 384:448] = centre_code(q0.float(), n_t)[:, None]
    y[:, 448:512] = torch.log10(torch.as_tensor(np.asarray(ps), dtype=torch.float32, device=fields.device))[:, None]
    return y, q0


def features(table, idx=None) -> np.ndarray:
    """Normalised network inputs [count][4] from a sweep table (n_thr, delta_rad, gdd_fs2, refl)."""
    raw = np.stack([np.asarray(table["n_thr"]), np.asarray(table["delta_rad"]), np.asarray(table["gdd_fs2"]),
                    np.asarray(table["refl"])], axis=1)
    if idx is not None:
        raw = raw[idx]
    return ((raw - FEAT_CENTER) / FEAT_HALF).astype(np.float32)


# ------------------------------------------------------------- the model

def _bias_mask(n_in: int, width: int, depth: int, n_out: int) -> np.ndarray:
    """True at the biases of the flat parameter layout (per layer W then b)."""
    parts = []
    for l in range(depth + 1):
        n = width if l < depth else n_out
        k = n_in if l == 0 else width
        parts += [np.zeros(n * k, bool), np.ones(n, bool)]
    return np.concatenate(parts)


class WarmStartModel:
    """The trained network plus its output scale (modes are stored divided by amp_scale)."""

    def __init__(self, mlp: MLP, amp_scale: float, meta: dict | None = None):
        self.mlp = mlp
        self.amp_scale = float(amp_scale)
        self.meta = dict(meta or {})
        self.kind = self.meta.get("kind", "low_modes")

    def save(self, path=MODEL_PATH) -> None:
        """Weights rounded to BF16 (the precision inference runs them at),
        stored as uint16; biases (added in FP32 by the epilogues) as float32."""
        p = self.mlp.get_params()
        bias = _bias_mask(self.mlp.n_in, self.mlp.width, self.mlp.depth, self.mlp.n_out)
        u = p[~bias].view(np.uint32).astype(np.uint64)
        u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
        Path(path).parent.mkdir(parents=True, exist_ok=True)
        np.savez_compressed(path, weights_bf16=u, biases=p[bias], amp_scale=self.amp_scale,
                            dims=np.array([self.mlp.n_in, self.mlp.width, self.mlp.depth, self.mlp.n_out]),
                            meta=np.array(repr(self.meta)))

    @staticmethod
    def load(path=MODEL_PATH, max_batch: int = 4096) -> "WarmStartModel":
        z = np.load(path)
        n_in, width, depth, n_out = (int(v) for v in z["dims"])
        mlp = MLP(n_in, width, depth, n_out, max_batch=max_batch)
        bias = _bias_mask(n_in, width, depth, n_out)
        p = np.zeros(bias.size, np.float32)
        p[~bias] = (z["weights_bf16"].astype(np.uint32) << 16).view(np.float32)
        p[bias] = z["biases"]
        mlp.set_params(p)
        meta = ast.literal_eval(str(z["meta"])) if "meta" in z else {}
        return WarmStartModel(mlp, float(z["amp_scale"]), meta)

    def predict_modes(self, feats):
        """Normalised features (numpy [count][4]) -> network outputs (CUDA float32 [count][512])."""
        torch = _torch()
        x = torch.from_numpy(np.ascontiguousarray(feats, np.float32)).cuda()
        return self.mlp.forward(x)

    def fields(self, pred, n_t: int, stream=None):
        """Network outputs -> initial signals (CUDA complex64 [count][n_t]) and the predicted powers."""
        torch = _torch()
        out = torch.empty(pred.shape[0], n_t, dtype=torch.complex64, device=pred.device)
        if self.kind == "band":
            check(load().cuopo_fields_from_bands(pred.contiguous().data_ptr(), pred.shape[0], n_t, 1.0,
                                                 out.data_ptr(), None, _stream(stream)))
            p0 = (10.0 ** pred[:, 448:512].double().mean(dim=1)).cpu().numpy()
        else:
            out = modes_to_fields(pred, n_t, self.amp_scale, stream=stream)
            # predicted power: mean |A|^2 = sum |c_q|^2 (Parseval)
            p0 = (self.amp_scale ** 2) * (pred.double() ** 2).sum(dim=1).cpu().numpy()
        return out, p0

    def close(self):
        self.mlp.close()


# ------------------------------------------------------------ data and training

def generate_data(count: int, seed: int, n_t: int = 8192, n_z: int = 100, max_rt: int = 5000, tol: float = 1e-7,
                  noise: float = 1e-15, kind: str = "band"):
    """Solves a uniformly drawn CW sweep at one grid size from noise (the
    plain batched solver) and returns the converged instances' features and
    training targets (band rows, or unscaled low-order modes), with the
    run's bookkeeping."""
    torch = _torch()
    from . import sweep
    base, insts, table = sweep.random_cw_sweep(count, seed, n_t_choices=(n_t,), n_z=n_z)
    t0 = time.perf_counter()
    with api.Batch(base, insts) as b:
        b.seed_noise(noise)
        b.run(max_rt, tol, 1)
        ps, rts, flags = b.results()
        sig = torch.empty(b.total, dtype=torch.complex64, device="cuda")
        b.get_signal(sig)
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    keep = np.flatnonzero((flags == 1) & (ps > 1e-20))
    conv = sig.reshape(count, n_t)[torch.from_numpy(keep).cuda()]
    if kind == "band":
        y, _ = band_targets(conv, ps[keep], n_t)
    else:
        y = fields_to_modes(conv, n_t)
    return {"x": features(table, keep), "y": y.cpu().numpy(), "ps": ps[keep], "rts": rts, "flags": flags,
            "seconds": secs, "count": count, "seed": seed, "n_t": n_t, "kind": kind}


def train(mlp: MLP, x: np.ndarray, y: np.ndarray, steps: int, batch: int = 4096, lr: float = 1e-3, seed: int = 0,
          log_every: int = 0):
    """Adam on (x, y) with minibatches drawn with replacement from the
    training set (a batch larger than the set repeats samples).  Returns the
    loss of every log_every-th step (device loss, read at the end)."""
    torch = _torch()
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    X = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    Y = torch.from_numpy(np.ascontiguousarray(y, np.float32)).cuda()
    n = X.shape[0]
    b = min(batch, mlp.max_batch)
    xb = torch.empty(b, X.shape[1], dtype=torch.float32, device="cuda")
    yb = torch.empty(b, Y.shape[1], dtype=torch.float32, device="cuda")
    losses = torch.zeros(max(1, steps), dtype=torch.float32, device="cuda")
    for s in range(steps):
        idx = torch.randint(0, n, (b,), generator=g, device="cuda")
        torch.index_select(X, 0, idx, out=xb)
        torch.index_select(Y, 0, idx, out=yb)
        # the learning rate drops 10x for the last 30 % of the steps
        mlp.train_step(xb, yb, lr if s < 0.7 * steps else 0.1 * lr, loss=losses[s])
    mlp.status()
    out = losses.cpu().numpy()
    return out if not log_every else out[::log_every]


def train_data_parallel(mlp, x: np.ndarray, y: np.ndarray, steps: int, batch: int = 4096, lr: float = 1e-3,
                        seed: int = 0, group=None):
    """Data-parallel Adam over the ranks of torch.distributed (one network
    copy per rank, NCCL on GPUs): rank r keeps the training rows r, r + W,
    ... and draws its minibatches from them; every step runs forward and
    backward on the rank's batch, sums the gradient buffers over the ranks
    (all-reduce on the current stream) and applies one Adam step with the
    mean.  `mlp` is any object with grad_step / grad_tensor / apply_adam
    (the MLP above).  Without an initialised process group it runs on one
    rank.  Returns this rank's per-step losses."""
    torch = _torch()
    import torch.distributed as dist
    on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if on else 1
    rank = dist.get_rank(group) if on else 0
    dev = mlp.grad_tensor().device
    X = torch.from_numpy(np.ascontiguousarray(x[rank::world], np.float32)).to(dev)
    Y = torch.from_numpy(np.ascontiguousarray(y[rank::world], np.float32)).to(dev)
    g = torch.Generator(device=dev)
    g.manual_seed(seed + 7919 * rank)
    n = X.shape[0]
    b = n if batch <= 0 or batch >= n else batch
    losses = torch.zeros(max(1, steps), dtype=torch.float32, device=dev)
    for s in range(steps):
        if b == n:
            xb, yb = X, Y
        else:
            idx = torch.randint(0, n, (b,), generator=g, device=dev)
            xb, yb = X.index_select(0, idx), Y.index_select(0, idx)
        mlp.grad_step(xb, yb, loss=losses[s])
        if world > 1:
            dist.all_reduce(mlp.grad_tensor(), op=dist.ReduceOp.SUM, group=group)
        mlp.apply_adam(lr if s < 0.7 * steps else 0.1 * lr, grad_scale=1.0 / world)
    return losses.cpu().numpy()


# ------------------------------------------------------------ warm-started solve

def warm_start(model: WarmStartModel, batch: "api.Batch", insts, table, noise: float = 1e-15,
               check_tol: float = 0.5, p_min: float = 1e-12, stream=None) -> dict:
    """Sets every instance's initial signal: the network's predicted steady
    state where it passes the first-round-trip check, else the instance's
    seeded noise (as a plain solve).  Leaves the batch reset at round trip 0.
    Returns per-instance acceptance and the predicted and checked powers."""
    torch = _torch()
    n_ts = np.array([x["n_t"] for x in insts])
    offs = np.concatenate([[0], np.cumsum(n_ts)])
    pred = model.predict_modes(features(table))
    sig_noise = torch.empty(batch.total, dtype=torch.complex64, device="cuda")
    batch.seed_noise(noise, stream=stream)
    batch.get_signal(sig_noise, stream=stream)
    trial = torch.empty_like(sig_noise)
    p0 = np.zeros(len(insts))
    for n in sorted(set(n_ts.tolist())):
        sel = np.flatnonzero(n_ts == n)
        f, p = model.fields(pred[torch.from_numpy(sel).cuda()], int(n), stream=stream)
        p0[sel] = p
        if np.all(np.diff(offs[sel]) == n) and len(sel) > 0:
            trial[offs[sel[0]]:offs[sel[-1] + 1]] = f.reshape(-1)
        else:
            for j, k in enumerate(sel):
                trial[offs[k]:offs[k + 1]] = f[j]
    batch.set_signal(trial, stream=stream)
    batch.reset(stream=stream)
    batch.step(1, 1, 0.0, 1, stream=stream)
    p1, _, _ = batch.results(stream=stream)
    resid = np.abs(p1 - p0) / np.maximum(p0, 1e-300)
    accept = (p0 > p_min) & (resid < check_tol)
    final = sig_noise.clone()
    for k in np.flatnonzero(accept):
        final[offs[k]:offs[k + 1]] = trial[offs[k]:offs[k + 1]]
    batch.set_signal(final, stream=stream)
    batch.reset(stream=stream)
    return {"accept": accept, "p0": p0, "p1": p1, "resid": resid}


def solve_sweep(base, insts, table, model: WarmStartModel | None, max_rt: int = 5000, tol: float = 1e-7,
                noise: float = 1e-15, check_tol: float = 0.5, return_fields: bool = False) -> dict:
    """One sweep solved to the convergence rule, from noise (model None) or
    warm-started; CUDA-event time of everything after batch creation
    (prediction, field synthesis, the check round trip, the solve)."""
    torch = _torch()
    st = torch.cuda.current_stream()
    with api.Batch(base, insts) as b:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        ws = None
        if model is None:
            b.seed_noise(noise)
            b.reset()
        else:
            ws = warm_start(model, b, insts, table, noise=noise, check_tol=check_tol)
        b.step(max_rt, max_rt, tol, 1)
        b.wait(st)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        ps, rts, flags = b.results()
        fields = None
        if return_fields:
            fields = torch.empty(b.total, dtype=torch.complex64, device="cuda")
            b.get_signal(fields)
    out = {"ms": ms, "ps": ps, "rts": rts, "flags": flags, "fields": fields}
    if ws is not None:
        out.update(accept=ws["accept"], resid=ws["resid"])
    return out


def _arm(r, count):
    conv = r["flags"] == 1
    n = int(np.sum(conv))
    out = {"seconds": r["ms"] * 1e-3, "converged": n, "round_trips": int(np.sum(r["rts"])),
           "solves_per_s": count / (r["ms"] * 1e-3), "converged_solves_per_s": n / (r["ms"] * 1e-3),
           "median_rts_converged": float(np.median(r["rts"][conv])) if n else None}
    if "accept" in r:
        acc = r["accept"]
        out.update(accepted=int(np.sum(acc)), accepted_converged=int(np.sum(acc & conv)),
                   median_rts_accepted_converged=float(np.median(r["rts"][acc & conv])) if np.any(acc & conv)
                   else None)
    return out


def _vs_plain(r, ref):
    both = (ref["flags"] == 1) & (r["flags"] == 1) & (ref["ps"] > 1e-20)
    err = np.abs(r["ps"][both] - ref["ps"][both]) / ref["ps"][both]
    return {"instances": int(np.sum(both)), "max_rel_err_ps": float(np.max(err)) if err.size else None,
            "median_rel_err_ps": float(np.median(err)) if err.size else None,
            "frac_within_1e-5": float(np.mean(err <= 1e-5)) if err.size else None}


def evaluate(model: WarmStartModel, count: int, seed: int, n_t: int = 8192, n_z: int = 100, max_rt: int = 5000,
             tol: float = 1e-7, check_tol: float = 0.5, control_noise: float = 1e-10) -> dict:
    """Held-out comparison on a freshly drawn sweep, the same instances,
    solver and rule in three arms: plain (noise-seeded, sigma 1e-15), warm
    (the network's prediction where it passes the first-round-trip check,
    else the same noise) and a control without the network (noise seeded
    with sigma `control_noise`, which also skips part of the build-up).  The
    final signal power of every instance that converged in an arm and in the
    plain solve is compared with the plain solve's."""
    from . import sweep
    base, insts, table = sweep.random_cw_sweep(count, seed, n_t_choices=(n_t,), n_z=n_z)
    plain = solve_sweep(base, insts, table, None, max_rt, tol)
    warm = solve_sweep(base, insts, table, model, max_rt, tol, check_tol=check_tol)
    ctrl = solve_sweep(base, insts, table, None, max_rt, tol, noise=control_noise) if control_noise else None
    conv_p = int(np.sum(plain["flags"] == 1))
    rate = lambda r: int(np.sum(r["flags"] == 1)) / r["ms"]
    out = {"count": count, "seed": seed, "n_t": n_t, "max_rt": max_rt, "tol": tol, "check_tol": check_tol,
           "model": model.kind, "plain": _arm(plain, count), "warm": _arm(warm, count),
           "gain_converged_solves_per_s": rate(warm) / rate(plain) if conv_p else None,
           "warm_vs_plain": _vs_plain(warm, plain)}
    if ctrl is not None:
        out["control_noise"] = control_noise
        out["control"] = _arm(ctrl, count)
        out["control_gain_converged_solves_per_s"] = rate(ctrl) / rate(plain) if conv_p else None
        out["control_vs_plain"] = _vs_plain(ctrl, plain)
    return out


def main():
    """python -m cuopo_b200.warmstart train|eval [options]: generates
    training data with the batched solver, trains the network on the GPU and
    writes the model (cuopo_b200/data/warmstart_mlp.npz) and a JSON summary."""
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "eval", "steps"],
                    help="train: data + training + held-out comparison; eval: comparison with the saved model; "
                         "steps: --steps training steps of a fresh network on random data (kernel timing and "
                         "profiling)")
    ap.add_argument("--count", type=int, default=4096, help="sweep instances solved for training data")
    ap.add_argument("--seed", type=int, default=100)
    ap.add_argument("--n-t", type=int, default=8192)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--eval-count", type=int, default=512)
    ap.add_argument("--eval-seed", type=int, default=7)
    ap.add_argument("--kind", choices=["band", "low_modes"], default="band")
    ap.add_argument("--save-data", type=str, default="", help="write the generated training set (npz)")
    ap.add_argument("--data", type=str, default="",
                    help="comma-separated saved training sets to train on (with --count > 0 a new set is also "
                         "generated and added)")
    ap.add_argument("--check-tol", type=float, default=0.5)
    ap.add_argument("--out", type=str, default=str(MODEL_PATH))
    ap.add_argument("--summary", type=str, default="")
    a = ap.parse_args()
    summary = {}
    if a.cmd == "steps":
        torch = _torch()
        mlp = MLP(max_batch=a.batch, seed=a.seed)
        x = torch.rand(a.batch, N_FEATURES, device="cuda") * 2 - 1
        t = torch.randn(a.batch, 2 * N_MODES, device="cuda")
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        for _ in range(a.steps):
            mlp.train_step(x, t, a.lr)
        ev[1].record()
        torch.cuda.synchronize()
        mlp.status()
        print(json.dumps({"steps": a.steps, "batch": a.batch, "ms_per_step": ev[0].elapsed_time(ev[1]) / a.steps}))
        return
    if a.cmd == "train":
        parts = []
        for path in [q for q in a.data.split(",") if q]:
            z = np.load(path)
            parts.append({k: z[k] for k in ("x", "y", "ps", "seconds")})
        if a.count > 0:
            g = generate_data(a.count, a.seed, n_t=a.n_t, kind=a.kind)
            if a.save_data:
                np.savez_compressed(a.save_data, x=g["x"], y=g["y"], ps=g["ps"], seconds=g["seconds"])
            parts.append(g)
        d = {"x": np.concatenate([q["x"] for q in parts]), "y": np.concatenate([q["y"] for q in parts]),
             "seconds": float(sum(float(q["seconds"]) for q in parts))}
        y = d["y"]
        if a.kind == "band":
            amp = 1.0
        else:
            # outputs scaled so that a typical steady state has unit norm over its modes
            amp = float(np.sqrt(np.mean(np.sum(y.astype(np.float64) ** 2, axis=1)))) if y.size else 1.0
        mlp = MLP(max_batch=a.batch, seed=a.seed)
        t0 = time.perf_counter()
        losses = train(mlp, d["x"], y / amp, a.steps, batch=a.batch, lr=a.lr, seed=a.seed)
        train_s = time.perf_counter() - t0
        model = WarmStartModel(mlp, amp, {"kind": a.kind, "sets": len(parts), "converged": int(len(y)),
                                          "seed": a.seed, "n_t": a.n_t, "steps": a.steps, "batch": a.batch,
                                          "lr": a.lr, "data_gpu_seconds": round(d["seconds"], 1)})
        model.save(a.out)
        summary.update(data={"sets": len(parts), "converged_states": int(len(y)), "seconds": d["seconds"],
                             "n_t": a.n_t},
                       train={"steps": a.steps, "batch": a.batch, "lr": a.lr, "seconds": train_s,
                              "loss_first": float(losses[0]), "loss_last": float(np.mean(losses[-50:]))},
                       amp_scale=amp)
    model = WarmStartModel.load(a.out)
    summary["eval"] = evaluate(model, a.eval_count, a.eval_seed, n_t=a.n_t, check_tol=a.check_tol)
    txt = json.dumps(summary, indent=1)
    print(txt)
    if a.summary:
        Path(a.summary).write_text(txt)


if __name__ == "__main__":
    main()
