"""Learned predictor stage of the xi step (no counterpart in the reference).

The reference's step (lcode.py:828-931) makes a first particle pass with the
PREVIOUS step's fields ("no halfstep-averaged fields yet", lcode.py:846-871)
only to obtain first-pass fields F1 for the corrector (lcode.py:876-901).
Here a small convolutional network (liblc3d's lc3d_predictor_*: 3x3
convolutions on the tcgen05 tensor cores, bf16 weights, fp32 accumulation)
predicts F1 from the fields of the two previous steps, and the step skips
the first pass's deposit and field solve (lc3d_step_arrays_predicted). The
corrector and final pass are the reference's; with a perfect prediction the
step is bit-identical to the plain one. The plain method judges the
network: every few steps a plain step also records its true first-pass
fields and the network's error against them; while that error is within the
tolerance the steps in between use the prediction, otherwise they run the
plain method (the fallback; run_learned).

Training data are the solver's own trajectories: lc3d_step_arrays_first_pass
returns F1 of every plain step, the target of the network; gradients and
Adam run in liblc3d's float32 training kernels.
"""
import ctypes
import time

import numpy as np
import torch

from . import _lib
from . import lcode as L
from ._lib import check, lib

FIELDS_IN = ('ro', 'jx', 'jy', 'jz', 'Ex', 'Ey', 'Bx', 'By', 'Bz')
FIELDS_OUT = ('Ex', 'Ey', 'Bx', 'By', 'Bz')
FIELDS_6 = ('Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz')
LAYERS = ((32, 32), (32, 64), (64, 128), (128, 64), (64, 32), (32, 16))   # (Cin, Cout) of conv1..conv6
N_IN, N_OUT = 27, 5   # used input channels (fields, differences, levels), outputs


def num_params():
    return int(lib.lc3d_predictor_num_params())


def init_params(seed, scale_last=0.1):
    """He-normal weights (fan-in 9 x used input channels), zero biases; the
    unused input channels of conv1 and outputs of conv6 are zero and conv6
    is scaled by ``scale_last``, so an untrained network predicts little
    more than linear extrapolation."""
    rng = np.random.default_rng(seed)
    out = []
    for k, (ci, co) in enumerate(LAYERS):
        ci_used = N_IN if k == 0 else ci
        w = rng.normal(0.0, np.sqrt(2.0 / (9 * ci_used)), size=(9, co, ci))
        if k == 0:
            w[:, :, N_IN:] = 0
        if k == len(LAYERS) - 1:
            w[:, N_OUT:, :] = 0
            w *= scale_last
        out += [w.ravel(), np.zeros(co)]
    return np.concatenate(out).astype(np.float32)


class _DeviceBuffer:
    """A raw device buffer as a torch tensor (no copy)."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {'shape': (count,), 'typestr': typestr, 'data': (ptr, False),
                                         'version': 2}


def _ptrs(tensors):
    return (ctypes.c_void_p * len(tensors))(*[t.data_ptr() for t in tensors])


class FieldPredictor:
    """One predictor instance for N x N grids on the current device."""

    def __init__(self, grid_steps, params=None, seed=0):
        self.N = int(grid_steps)
        self.device = L._device()
        self.h = ctypes.c_void_p()
        check(lib.lc3d_predictor_create(self.N, self.device.index, ctypes.byref(self.h)), 'lc3d_predictor_create')
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        self.set_params(init_params(seed) if params is None else params)
        self._buf = {}
        for name, which, typ in (('input', _lib.PRED_INPUT, '<i2'), ('output', _lib.PRED_OUTPUT, '<f4'),
                                 ('target', _lib.PRED_TARGET, '<f4')):
            p, nb = ctypes.c_void_p(), ctypes.c_longlong()
            check(lib.lc3d_predictor_tensor(self.h, which, ctypes.byref(p), ctypes.byref(nb)), 'lc3d_predictor_tensor')
            item = 2 if typ == '<i2' else 4
            self._buf[name] = torch.as_tensor(_DeviceBuffer(p.value, nb.value // item, typ), device=self.device)

    def __del__(self):
        h = getattr(self, 'h', None)
        if h is not None and h.value and lib is not None:
            lib.lc3d_predictor_destroy(h)
            self.h = None

    # -- parameters -------------------------------------------------------
    def set_params(self, params):
        t = torch.as_tensor(np.asarray(params, np.float32) if not torch.is_tensor(params) else params,
                            dtype=torch.float32).to(self.device).contiguous()
        assert t.numel() == num_params()
        check(lib.lc3d_predictor_set_params(self.h, ctypes.c_void_p(t.data_ptr()), L._stream()), 'set_params')
        torch.cuda.current_stream().synchronize()

    def params(self):
        t = torch.empty(num_params(), dtype=torch.float32, device=self.device)
        check(lib.lc3d_predictor_get_params(self.h, ctypes.c_void_p(t.data_ptr()), L._stream()), 'get_params')
        return t

    def grad(self):
        t = torch.empty(num_params(), dtype=torch.float32, device=self.device)
        check(lib.lc3d_predictor_get_grad(self.h, ctypes.c_void_p(t.data_ptr()), L._stream()), 'get_grad')
        return t

    def set_scales(self, in_mult, out_mult):
        a = (ctypes.c_double * 18)(*[float(v) for v in in_mult])
        b = (ctypes.c_double * 5)(*[float(v) for v in out_mult])
        check(lib.lc3d_predictor_set_scales(self.h, a, b), 'set_scales')

    def buffer(self, name):
        """The device buffer 'input' (bf16 bits as int16), 'output' or
        'target' (float32) as a flat torch tensor view."""
        return self._buf[name]

    # -- inference ----------------------------------------------------------
    def pack(self, f1, f2):
        """Network input from the fields (objects with the FIELDS_IN
        attributes, N x N float64 device tensors) of steps t-1 and t-2."""
        a = _ptrs([getattr(f1, n) for n in FIELDS_IN])
        b = _ptrs([getattr(f2, n) for n in FIELDS_IN])
        check(lib.lc3d_predictor_pack(self.h, a, b, L._stream()), 'lc3d_predictor_pack')

    def forward(self):
        check(lib.lc3d_predictor_forward(self.h, L._stream()), 'lc3d_predictor_forward')

    def predict_into(self, f1, f2, out):
        """pack + forward + predictions of Ex, Ey, Bx, By, Bz (and Ez by
        linear extrapolation) into out (a dict of N x N float64 device
        tensors)."""
        self.pack(f1, f2)
        self.forward()
        check(lib.lc3d_predictor_predict(self.h, _ptrs([getattr(f1, n) for n in FIELDS_6]),
                                         _ptrs([getattr(f2, n) for n in FIELDS_6]),
                                         _ptrs([out[n] for n in FIELDS_6]), L._stream()), 'predict')

    # -- training -------------------------------------------------------------
    def set_target(self, first, f1, f2):
        check(lib.lc3d_predictor_set_target(self.h, _ptrs([first[n] for n in FIELDS_6]),
                                            _ptrs([getattr(f1, n) for n in FIELDS_6]),
                                            _ptrs([getattr(f2, n) for n in FIELDS_6]), L._stream()),
              'set_target')

    def backward(self):
        """Gradients of the MSE on the current input / target (after
        forward); the loss is added to ``self.loss``."""
        check(lib.lc3d_predictor_backward(self.h, ctypes.c_void_p(self.loss.data_ptr()), L._stream()), 'backward')

    def adam(self, lr):
        check(lib.lc3d_predictor_adam(self.h, ctypes.c_float(lr), L._stream()), 'adam')

    def check_errors(self):
        check(lib.lc3d_predictor_check_error(self.h, L._stream()), 'predictor')

    def save(self, path):
        np.savez(path, params=self.params().cpu().numpy(), grid_steps=self.N)

    @classmethod
    def load(cls, path, grid_steps=None):
        d = np.load(path)
        return cls(int(grid_steps or d['grid_steps']), params=d['params'])


# ---------------------------------------------------------------------------
# Trajectories of the solver (training data)
# ---------------------------------------------------------------------------

def _state_buffers(config, like):
    g = (config.grid_steps,) * 2
    shape_p = tuple(like.x_offt.shape)
    st = L.GPUArrays.__new__(L.GPUArrays)
    for k, n in enumerate(_lib.STATE_NAMES):
        setattr(st, n, L._empty(shape_p if k < 5 else g))
    return st


def _sp(st):
    return _lib.StatePtrs(*[getattr(st, n).data_ptr() for n in _lib.STATE_NAMES])


class Stepper:
    """Host loop of one simulation on caller-owned state buffers: plain,
    first-pass-recording and predicted steps with the device beam."""

    def __init__(self, config, beam, xi0=0):
        self.config = config
        self.xs, self.ys, self.const, self.virt, state = L.init(config)
        self.solver = L.solver_for(config)
        self.solver.set_virt(self.virt)
        self.solver.set_const(self.const)
        bp = _lib.BeamParams(*[float(v) for v in beam])
        check(lib.lc3d_set_beam(self.solver.ctx, ctypes.byref(bp)), 'lc3d_set_beam')
        self.bufs = [_state_buffers(config, state) for _ in range(3)]
        for n in _lib.STATE_NAMES:
            getattr(self.bufs[0], n).copy_(L._f64(getattr(state, n)))
        self.cur, self.prev = 0, None     # indices into bufs: state t-1, state t-2
        self.xi = xi0
        N = config.grid_steps
        self.beam = L._empty((N, N))
        self.first = {n: L._empty((N, N)) for n in FIELDS_6}
        self.pred = {n: L._empty((N, N)) for n in FIELDS_6}
        self.residual = L._empty((1,))
        self.error = L._empty((1,))

    @property
    def state(self):
        return self.bufs[self.cur]

    @property
    def state_prev(self):
        return None if self.prev is None else self.bufs[self.prev]

    def _out(self):
        used = {self.cur, self.prev}
        return next(k for k in range(3) if k not in used)

    def _beam(self):
        check(lib.lc3d_beam_eval(self.solver.ctx, self.xi, ctypes.c_void_p(self.beam.data_ptr()), L._stream()),
              'lc3d_beam_eval')

    def _advance(self, o):
        self.prev, self.cur = self.cur, o
        self.xi += 1

    def step_plain(self, record_first=False):
        o = self._out()
        self._beam()
        if record_first:
            firsts = (ctypes.c_void_p * 6)(*[self.first[n].data_ptr() for n in FIELDS_6])
            check(lib.lc3d_step_arrays_first_pass(self.solver.ctx, ctypes.byref(_sp(self.state)),
                                                  ctypes.byref(_sp(self.bufs[o])),
                                                  ctypes.c_void_p(self.beam.data_ptr()), firsts, L._stream()),
                  'first-pass step')
        else:
            check(lib.lc3d_step_arrays(self.solver.ctx, ctypes.byref(_sp(self.state)), ctypes.byref(_sp(self.bufs[o])),
                                       ctypes.c_void_p(self.beam.data_ptr()), L._stream()), 'step')
        self._advance(o)

    def step_predicted(self, predictor, residual=False):
        """One step with the network's prediction in place of the first
        pass (lc3d_step_arrays_predicted). With ``residual`` the corrector's
        change of the prediction is left in ``self.residual``."""
        f1, f2 = self.state, self.state_prev
        predictor.predict_into(f1, f2, self.pred)
        o = self._out()
        self._beam()
        preds = (ctypes.c_void_p * 6)(*[self.pred[n].data_ptr() for n in FIELDS_6])
        check(lib.lc3d_step_arrays_predicted(self.solver.ctx, ctypes.byref(_sp(self.state)),
                                             ctypes.byref(_sp(self.bufs[o])), ctypes.c_void_p(self.beam.data_ptr()),
                                             preds, ctypes.c_void_p(self.residual.data_ptr()) if residual else None,
                                             L._stream()), 'predicted step')
        self._advance(o)

    def step_verify(self, predictor):
        """A plain step that records the true first-pass fields F1, with the
        network's prediction for the same step; leaves max|pred - F1| /
        max|F1| over Ex, Ey, Bx, By, Bz in ``self.error`` (device)."""
        predictor.predict_into(self.state, self.state_prev, self.pred)
        self.step_plain(record_first=True)
        a = (ctypes.c_void_p * 6)(*[self.pred[n].data_ptr() for n in FIELDS_6])
        b = (ctypes.c_void_p * 6)(*[self.first[n].data_ptr() for n in FIELDS_6])
        check(lib.lc3d_fields_rel_diff(self.solver.ctx, a, b, ctypes.c_void_p(self.error.data_ptr()), L._stream()),
              'lc3d_fields_rel_diff')
        return self.error


class Sample:
    """One training sample kept on the device: the packed network input
    (bf16 bits) and the target (float32)."""

    def __init__(self, x, t):
        self.x, self.t = x, t


def generate_samples(predictor, config, beam, nsteps, every=1, start=2):
    """Run ``nsteps`` plain steps recording the first-pass fields; from step
    ``start`` on, every ``every``-th step becomes a sample. Returns (list of
    Sample, Ez(N/2, N/2) history as numpy)."""
    sim = Stepper(config, beam)
    N = config.grid_steps
    out, ez = [], []
    for i in range(nsteps):
        take = i >= start and (i - start) % every == 0
        f1, f2 = sim.state, sim.state_prev
        sim.step_plain(record_first=take)
        if take:
            predictor.pack(f1, f2)
            predictor.set_target(sim.first, f1, f2)
            out.append(Sample(predictor.buffer('input').clone(), predictor.buffer('target').clone()))
        ez.append(sim.state.Ez[N // 2, N // 2].clone())
    return out, torch.stack(ez).cpu().numpy()


def train(predictor, samples, epochs, lr=1e-3, seed=0, lr_final=None, log=None):
    """Adam over the samples (batch of one, shuffled each epoch, cosine
    learning-rate decay to ``lr_final``). Returns the mean loss per epoch."""
    rng = np.random.default_rng(seed)
    lr_final = lr * 0.05 if lr_final is None else lr_final
    total = epochs * len(samples)
    xin, tin = predictor.buffer('input'), predictor.buffer('target')
    hist, k = [], 0
    for ep in range(epochs):
        predictor.loss.zero_()
        for i in rng.permutation(len(samples)):
            s = samples[int(i)]
            xin.copy_(s.x)
            tin.copy_(s.t)
            predictor.forward()
            predictor.backward()
            a = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * k / max(total - 1, 1)))
            predictor.adam(float(a))
            k += 1
        hist.append(float(predictor.loss.item()) / len(samples))
        if log:
            log(f'epoch {ep}: loss {hist[-1]:.4e}')
    predictor.check_errors()
    return hist


def evaluate(predictor, samples):
    """Mean loss of the network (and of the untrained baseline: zero
    output, i.e. linear extrapolation) over samples."""
    xin, tin = predictor.buffer('input'), predictor.buffer('target')
    net, base = 0.0, 0.0
    for s in samples:
        xin.copy_(s.x)
        tin.copy_(s.t)
        predictor.forward()
        y = predictor.buffer('output').view(-1, 16)[:, :N_OUT]
        t = s.t.view(-1, 16)[:, :N_OUT]
        net += float(((y - t) ** 2).mean())
        base += float((t ** 2).mean())
    return net / len(samples), base / len(samples)


def learned_steps(sim, predictor, nsteps, tol=1e-6, verify_every=10, warm=0, record=True):
    """Advance ``sim`` (a Stepper) by ``nsteps`` steps with the learned first
    pass under periodic verification: the first ``warm`` steps are plain,
    then every ``verify_every``-th step is a plain step that also checks the
    network against that step's true first-pass fields
    (Stepper.step_verify); while the last check's error max|pred - F1| /
    max|F1| is within ``tol`` the steps in between use the prediction,
    otherwise they are plain (the fallback). Returns (list of Ez(N/2, N/2)
    device scalars, or [] without ``record``; counters)."""
    N = sim.config.grid_steps
    ez, errs = [], []
    n_learned = n_plain = n_verify = n_fail = 0
    use = False
    for i in range(nsteps):
        if i < warm:
            sim.step_plain()
            n_plain += 1
        elif (i - warm) % verify_every == 0:
            e = float(sim.step_verify(predictor).item())
            errs.append(e)
            n_verify += 1
            use = e <= tol
            n_fail += int(not use)
        elif use:
            sim.step_predicted(predictor)
            n_learned += 1
        else:
            sim.step_plain()
            n_plain += 1
        if record:
            ez.append(sim.state.Ez[N // 2, N // 2].clone())
    stats = {'steps': nsteps, 'learned_steps': n_learned, 'plain_steps': n_plain, 'verify_steps': n_verify,
             'first_passes_saved': n_learned, 'fallback_rate': (n_fail / n_verify) if n_verify else None,
             'pred_err_median': float(np.median(errs)) if errs else None,
             'pred_err_max': float(np.max(errs)) if errs else None, 'tol': tol, 'verify_every': verify_every}
    return ez, stats


def run_learned(config, beam, nsteps, predictor, tol=1e-6, verify_every=10, warm=20, record=True):
    """Run ``nsteps`` steps from the initial state (learned_steps after
    ``warm`` plain steps). Returns (Ez(N/2, N/2) history or None, stats, the
    Stepper)."""
    sim = Stepper(config, beam)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ez, stats = learned_steps(sim, predictor, nsteps, tol, verify_every, warm, record)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    stats['wall_s'] = wall
    stats['xi_steps_per_s'] = nsteps / wall
    return (torch.stack(ez).cpu().numpy() if record else None), stats, sim


def draw_beams(count, seed, amp=(0.01, 0.5), sigma=(0.7, 1.5)):
    """Seeded beam draws: amplitude log-uniform, sigma_r uniform, length
    factor 1."""
    rng = np.random.default_rng(seed)
    return [(float(np.exp(rng.uniform(np.log(amp[0]), np.log(amp[1])))), float(rng.uniform(*sigma)), 1.0)
            for _ in range(count)]


def train_streaming(predictor, make_cfg, beams, nsteps, every=30, start=20, buffer=600, lr=1e-3, lr_final=5e-5,
                    epochs_per_run=1, seed=0, log=None):
    """Train on solver runs as they are generated: each run's samples join a
    replay buffer (oldest dropped beyond ``buffer``) and the network makes
    ``epochs_per_run`` passes over the buffer at a learning rate that decays
    (cosine) from ``lr`` to ``lr_final`` over the runs. Returns the mean
    loss of each pass."""
    buf, hist = [], []
    n = len(beams)
    for k, b in enumerate(beams):
        smp, _ = generate_samples(predictor, make_cfg(b), b, nsteps, every=every, start=start)
        buf += smp
        if len(buf) > buffer:
            buf = buf[len(buf) - buffer:]
        a = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * k / max(n - 1, 1)))
        h = train(predictor, buf, epochs_per_run, lr=a, lr_final=a, seed=seed + k)
        hist += h
        if log:
            log(f'run {k + 1}/{n} beam {b}: {len(smp)} samples, buffer {len(buf)}, lr {a:.2e}, loss {h[-1]:.4e}')
    return hist
