"""The learned develop: a small convolutional surrogate of the plain develop,
run and trained on the device by the library's own kernels (learned.cu).

`Surrogate` holds the f32 parameters and the noise range the network was
trained on; `develop_learned` / `develop_learned_planar_into` develop a
decoded Frame with it (tiles whose noise channel leaves the trained range
fall back to the plain develop); `Trainer` and `train_surrogate` train it on
crops of frames developed by the plain GPU path.
"""

from __future__ import annotations

import ctypes as C
import dataclasses
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from . import (DemosaicParams, Error, Frame, RgbPlanes, Stage, _check, _dptr, _error, _torch, context,
               frame_quantizer)

# Layer shapes (cin, cout) of the network, head last.
LAYERS = [(16, 32)] + [(32, 32)] * 5 + [(32, 16)]
HEAD_USED = 12


def param_count() -> int:
    return int(_lib.lib().prr_sg_param_count())


def layer_slices():
    """(weights, bias) slices of each layer in the flat parameter vector."""
    out, off = [], 0
    for cin, cout in LAYERS:
        nw = cout * cin * 9
        out.append((slice(off, off + nw), slice(off + nw, off + nw + cout)))
        off += nw + cout
    return out


@dataclasses.dataclass
class Surrogate:
    params: np.ndarray  # f32, param_count()
    noise_lo: float = 0.0
    noise_hi: float = float("inf")

    @staticmethod
    def init(seed: int = 0, scale: float = 1.0) -> "Surrogate":
        """He-normal weights, zero biases; the head starts at zero so that the
        untrained network outputs each quad's own colour."""
        rng = np.random.default_rng(seed)
        p = np.zeros(sum(cout * cin * 9 + cout for cin, cout in LAYERS), dtype=np.float32)
        for k, ((cin, cout), (ws, bs)) in enumerate(zip(LAYERS, layer_slices())):
            if k == len(LAYERS) - 1:
                continue
            p[ws] = rng.normal(0.0, scale * np.sqrt(2.0 / (cin * 9)), ws.stop - ws.start).astype(np.float32)
        return Surrogate(p)

    def save(self, path: str) -> None:
        np.savez(path, params=self.params, noise=np.array([self.noise_lo, self.noise_hi], dtype=np.float32))

    @staticmethod
    def load(path: str) -> "Surrogate":
        z = np.load(path)
        return Surrogate(z["params"].astype(np.float32), float(z["noise"][0]), float(z["noise"][1]))

    def device(self):
        torch = _torch()
        return torch.from_numpy(np.ascontiguousarray(self.params, dtype=np.float32)).cuda()


DEFAULT_MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "surrogate.npz")


def default_surrogate() -> Surrogate:
    """The packaged network: trained by this library on 4000 512x512 crops
    of synthetic 4096x2160 frames (noise sigma 4..32, qscale 15..45)."""
    return Surrogate.load(DEFAULT_MODEL)


def _model(s: Surrogate, dev_params) -> _lib.CSgModel:
    return _lib.CSgModel(dev_params.data_ptr(), float(s.noise_lo), float(s.noise_hi))


def develop_learned_planar_into(frame: Frame, params: DemosaicParams, stage: Stage, surrogate: Surrogate,
                                out: Sequence, dev_params=None, count_fallback: bool = True) -> int:
    """develop_planar_into by the surrogate; returns the number of 32x32
    tiles developed by the plain fallback (count_fallback False: returns -1
    and does not wait for the device, so the call can be captured in a CUDA
    graph)."""
    torch = _torch()
    n = frame.header.width * frame.header.height
    if len(out) != 3 or any(int(o.numel()) != n for o in out):
        raise Error(_lib.ERR_BUFFER, message="plane size")
    dp = dev_params if dev_params is not None else surrogate.device()
    ctx = context()
    m = _model(surrogate, dp)
    nfb = C.c_uint32()
    rc = _lib.lib().prr_develop_learned(ctx, C.byref(frame.header._c), C.byref(params._c()), int(stage),
                                        _dptr(frame.samples), C.byref(m), 1, _dptr(out[0]), _dptr(out[1]),
                                        _dptr(out[2]), n, C.byref(nfb) if count_fallback else None)
    _check(rc, ctx=ctx)
    return int(nfb.value) if count_fallback else -1


def develop_learned(frame: Frame, stage: Stage, surrogate: Surrogate,
                    params: Optional[DemosaicParams] = None) -> Tuple[RgbPlanes, int]:
    """develop_planar with the surrogate: (planes, fallback tiles)."""
    torch = _torch()
    if params is None:
        params = DemosaicParams.new(frame.header, frame.quantizer())
    n = frame.header.width * frame.header.height
    planes = torch.empty(3 * n, dtype=torch.float32, device="cuda")
    r, g, b = planes[:n], planes[n:2 * n], planes[2 * n:]
    nfb = develop_learned_planar_into(frame, params, stage, surrogate, [r, g, b])
    return RgbPlanes(frame.header.width, frame.header.height, [r, g, b]), nfb


def pack(frame: Frame, stage: Stage, params: Optional[DemosaicParams] = None) -> Tuple[np.ndarray, np.ndarray]:
    """prr_sg_pack: the network input [16][hq][wq] and the quad colours
    [3][hq][wq] the learned develop computes for a decoded frame (checking)."""
    if params is None:
        params = DemosaicParams.new(frame.header, frame.quantizer())
    hq, wq = (frame.header.height + 1) // 2, (frame.header.width + 1) // 2
    in16 = np.zeros((16, hq, wq), dtype=np.float32)
    base = np.zeros((3, hq, wq), dtype=np.float32)
    ctx = context()
    rc = _lib.lib().prr_sg_pack(ctx, C.byref(frame.header._c), C.byref(params._c()), int(stage),
                                _dptr(frame.samples), in16.ctypes.data, base.ctypes.data)
    _check(rc, ctx=ctx)
    return in16, base


def gradients(in16: np.ndarray, base3: np.ndarray, target3: np.ndarray, params: np.ndarray):
    """Device forward, loss and gradient for one explicit image (checking)."""
    hq, wq = in16.shape[1:]
    head = np.zeros((16, hq, wq), dtype=np.float32)
    dp = np.zeros(param_count(), dtype=np.float32)
    loss = C.c_double()
    ctx = context()
    a = [np.ascontiguousarray(x, dtype=np.float32) for x in (in16, base3, target3, params)]
    rc = _lib.lib().prr_sg_gradients(ctx, a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, hq, wq,
                                     a[3].ctypes.data, head.ctypes.data, dp.ctypes.data, C.byref(loss))
    _check(rc, ctx=ctx)
    return head, dp, float(loss.value)


class Trainer:
    """prr_sg_trainer: frames (decoded, with their plain develop as target)
    and Adam state on the device."""

    def __init__(self, batch: int = 32, crop: int = 512):
        self.ctx = context()
        self.batch, self.crop = batch, crop
        self.t = C.c_void_p()
        _check(_lib.lib().prr_sg_trainer_create(self.ctx, batch, crop, C.byref(self.t)), ctx=self.ctx)
        self.frames: List[Tuple[int, int]] = []

    def close(self):
        if self.t:
            _lib.lib().prr_sg_trainer_destroy(self.t)
            self.t = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_frame(self, frame: Frame, params: Optional[DemosaicParams] = None) -> int:
        if params is None:
            params = DemosaicParams.new(frame.header, frame.quantizer())
        idx = C.c_uint32()
        _check(_lib.lib().prr_sg_trainer_add_frame(self.t, C.byref(frame.header._c), C.byref(params._c()),
                                                  _dptr(frame.samples), C.byref(idx)), ctx=self.ctx)
        self.frames.append((frame.header.width, frame.header.height))
        return int(idx.value)

    def noise_range(self) -> Tuple[float, float]:
        lo, hi = C.c_float(), C.c_float()
        _check(_lib.lib().prr_sg_trainer_noise_range(self.t, C.byref(lo), C.byref(hi)), ctx=self.ctx)
        return float(lo.value), float(hi.value)

    def set_params(self, p: np.ndarray) -> None:
        a = np.ascontiguousarray(p, dtype=np.float32)
        _check(_lib.lib().prr_sg_trainer_set_params(self.t, a.ctypes.data), ctx=self.ctx)

    def get_params(self) -> np.ndarray:
        a = np.zeros(param_count(), dtype=np.float32)
        _check(_lib.lib().prr_sg_trainer_get_params(self.t, a.ctypes.data), ctx=self.ctx)
        return a

    def random_crops(self, rng: np.random.Generator) -> np.ndarray:
        crops = np.zeros((self.batch, 3), dtype=np.uint32)
        for k in range(self.batch):
            f = int(rng.integers(len(self.frames)))
            w, h = self.frames[f]
            crops[k] = (f, 2 * int(rng.integers((w - self.crop) // 2 + 1)),
                        2 * int(rng.integers((h - self.crop) // 2 + 1)))
        return crops

    def step(self, crops: np.ndarray, lr: float, want_loss: bool = True) -> Optional[float]:
        a = np.ascontiguousarray(crops, dtype=np.uint32)
        loss = C.c_float()
        rc = _lib.lib().prr_sg_trainer_step(self.t, a.ctypes.data, float(lr),
                                            C.byref(loss) if want_loss else None)
        _check(rc, ctx=self.ctx)
        return float(loss.value) if want_loss else None


def train_surrogate(frames: Sequence[Frame], crops: int = 4000, batch: int = 32, crop: int = 512,
                    epochs: int = 8, lr: float = 1e-3, seed: int = 0, log=None) -> Tuple[Surrogate, List[float]]:
    """Train on `crops` random crops of the frames (drawn once, seeded),
    `epochs` passes of Adam with the given learning rate (cosine decay to
    a tenth over the run)."""
    tr = Trainer(batch, crop)
    for f in frames:
        tr.add_frame(f)
    s = Surrogate.init(seed)
    tr.set_params(s.params)
    rng = np.random.default_rng(seed)
    pool = np.concatenate([tr.random_crops(rng) for _ in range((crops + batch - 1) // batch)])[:crops]
    steps_per_epoch = max(1, len(pool) // batch)
    total = steps_per_epoch * epochs
    history = []
    k = 0
    for ep in range(epochs):
        order = rng.permutation(len(pool))
        for i in range(steps_per_epoch):
            sel = pool[order[i * batch:(i + 1) * batch]]
            lr_k = lr * (0.1 + 0.9 * 0.5 * (1.0 + np.cos(np.pi * k / total)))
            want = (i == steps_per_epoch - 1)
            loss = tr.step(sel, lr_k, want_loss=want)
            if want:
                history.append(loss)
                if log:
                    log(f"epoch {ep} loss {loss:.3e}")
            k += 1
    s.params = tr.get_params()
    s.noise_lo, s.noise_hi = tr.noise_range()
    tr.close()
    return s, history


def psnr(a: np.ndarray, b: np.ndarray, peak: float = 1.0) -> float:
    mse = float(np.mean((np.asarray(a, dtype=np.float64) - np.asarray(b, dtype=np.float64)) ** 2))
    return float("inf") if mse == 0 else 10.0 * np.log10(peak * peak / mse)


def max_abs(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.max(np.abs(np.asarray(a, dtype=np.float64) - np.asarray(b, dtype=np.float64))))


def _main(argv=None) -> int:
    """Develop a synthetic frame with the packaged network and time it:
    python -m proresraw_rs_b200.learned [--width W] [--height H] [--reps N]"""
    import argparse
    import time

    from . import synth as S

    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=4096)
    ap.add_argument("--height", type=int, default=2160)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--seed", type=int, default=7)
    a = ap.parse_args(argv)
    torch = _torch()
    from . import decode_frame, develop_planar_into

    m = S.mosaic(a.width, a.height, S.RGGB, seed=a.seed, sigma=16.0, white=4095)
    spec = S.Spec(a.width, a.height, pattern=S.RGGB, alignment=2, white_level=4095, valid_tiles=True, wb=(1.9, 1.4),
                  color_matrix=(0.61, 0.25, 0.10, 0.26, 0.89, -0.15, 0.02, -0.09, 1.17))
    f = decode_frame(S.encode(spec, m, qscale=30, qscale_seed=a.seed))
    s = default_surrogate()
    n = a.width * a.height
    out = [torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(3)]
    prm = DemosaicParams.new(f.header, f.quantizer())
    dp = s.device()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    develop_learned_planar_into(f, prm, Stage.REC2020, s, out, dev_params=dp)
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(a.reps):
        develop_learned_planar_into(f, prm, Stage.REC2020, s, out, dev_params=dp, count_fallback=False)
    ev[1].record()
    for _ in range(a.reps):
        develop_planar_into(f, prm, Stage.REC2020, out)
    ev[2].record()
    torch.cuda.synchronize()
    print(f"{a.width}x{a.height}: learned develop {ev[0].elapsed_time(ev[1]) / a.reps:.3f} ms, "
          f"plain develop {ev[1].elapsed_time(ev[2]) / a.reps:.3f} ms")
    return 0


if __name__ == "__main__":
    raise SystemExit(_main())
