"""Train the learned field predictor on the solver's own trajectories and
save its parameters (python -m lcode3d_b200.train_predictor).

Training runs: seeded draws of the axisymmetric driver (amplitude
log-uniform on [0.01, 0.5], sigma_r uniform on [0.7, 1.5]) at the
production grid (641 x 641, h = 0.025, xi_step = 0.005); each run's
first-pass fields are the targets (lc3d_step_arrays_first_pass). Held-out
runs (another seed) evaluate the network (mean squared error of the
first-pass correction against linear extrapolation) and the learned method
under periodic verification at the given tolerances (Ez(N/2, N/2) against
the plain method over the same steps). Writes the parameters as .npz and a
JSON summary.
"""
import argparse
import json
import os
import sys
import time
import types

import numpy as np

from . import predictor as P

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, 'data', 'field_predictor_641.npz')


def make_config(N, h, dxi, nsteps):
    """A config object with the reference's attribute names (the beam is
    given to the solver by its parameters, not by config.beam)."""
    def mk(beam):
        return types.SimpleNamespace(
            grid_steps=N, grid_step_size=h, xi_step_size=dxi, xi_steps=nsteps, diagnostics_each_N_steps=10 ** 9,
            field_solver_subtraction_trick=1, field_solver_variant_A=True, reflect_padding_steps=5,
            plasma_padding_steps=10, plasma_coarseness=3, plasma_fineness=2, gpu_index=0)
    return mk


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument('--grid', type=int, default=641)
    ap.add_argument('--h', type=float, default=0.025)
    ap.add_argument('--xi-step', type=float, default=0.005)
    ap.add_argument('--steps', type=int, default=3000, help='xi steps per run')
    ap.add_argument('--runs', type=int, default=200, help='training runs')
    ap.add_argument('--held-out', type=int, default=20)
    ap.add_argument('--eval-runs', type=int, default=20, help='held-out runs of the learned method')
    ap.add_argument('--every', type=int, default=30)
    ap.add_argument('--buffer', type=int, default=600)
    ap.add_argument('--epochs-per-run', type=int, default=2)
    ap.add_argument('--lr', type=float, default=1e-3)
    ap.add_argument('--seed', type=int, default=1)
    ap.add_argument('--tols', default='1e-6,1e-4')
    ap.add_argument('--out', default=DEFAULT_WEIGHTS)
    ap.add_argument('--summary', default=None)
    a = ap.parse_args(argv)
    mk = make_config(a.grid, a.h, a.xi_step, a.steps)
    pr = P.FieldPredictor(a.grid, seed=a.seed)
    t0 = time.time()
    hist = P.train_streaming(pr, mk, P.draw_beams(a.runs, a.seed), a.steps, every=a.every, buffer=a.buffer,
                             lr=a.lr, epochs_per_run=a.epochs_per_run, seed=a.seed,
                             log=lambda m: print(m, flush=True))
    t_train = time.time() - t0
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    pr.save(a.out)
    held = P.draw_beams(a.held_out, a.seed + 1000)
    ev = []
    for b in held:
        smp, _ = P.generate_samples(pr, mk(b), b, a.steps, every=a.every * 5 + 1, start=20)
        ev.append(P.evaluate(pr, smp))
        del smp
    net = float(np.mean([e[0] for e in ev]))
    base = float(np.mean([e[1] for e in ev]))
    print(f'held-out ({len(held)} runs): MSE network {net:.4e}, linear extrapolation {base:.4e}, '
          f'ratio {net / base:.4e}', flush=True)
    learned, table = [], {}
    for tol in [float(t) for t in a.tols.split(',')]:
        rows = []
        for b in held[:a.eval_runs]:
            cfg = mk(b)
            ez_l, st, _ = P.run_learned(cfg, b, a.steps, pr, tol=tol)
            ez_p, stp, _ = P.run_learned(cfg, b, a.steps, pr, tol=-1.0)   # plain steps only
            st['tol'] = tol
            st['beam'] = b
            st['ez_max_rel_err_vs_plain'] = float(np.abs(ez_l - ez_p).max() / np.abs(ez_p).max())
            st['plain_xi_steps_per_s'] = stp['xi_steps_per_s']
            learned.append(st)
            rows.append(st)
            print(json.dumps(st), flush=True)
        # the config's report over the held-out seeds: first passes saved,
        # fallback rate, Ez error against the float64 method, speed
        table[f'{tol:g}'] = {
            'runs': len(rows),
            'first_passes_saved_mean': float(np.mean([r['learned_steps'] / a.steps for r in rows])),
            'fallback_rate_mean': float(np.mean([1.0 if r['fallback_rate'] is None else r['fallback_rate']
                                                 for r in rows])),
            'ez_max_rel_err_vs_fp64_max': float(np.max([r['ez_max_rel_err_vs_plain'] for r in rows])),
            'xi_steps_per_s_mean': float(np.mean([r['xi_steps_per_s'] for r in rows])),
            'plain_xi_steps_per_s_mean': float(np.mean([r['plain_xi_steps_per_s'] for r in rows])),
        }
        print(json.dumps({'tol': tol, **table[f'{tol:g}']}), flush=True)
    summary = {'grid': a.grid, 'runs': a.runs, 'steps_per_run': a.steps, 'every': a.every,
               'epochs_per_run': a.epochs_per_run, 'train_seconds': t_train, 'loss_history': hist,
               'held_out_runs': len(held), 'held_out_mse_network': net, 'held_out_mse_linear_extrapolation': base,
               'learned_runs': learned, 'learned_table': table,
               'weights': os.path.relpath(a.out, os.path.dirname(HERE))}
    if a.summary:
        with open(a.summary, 'w') as f:
            json.dump(summary, f, indent=1)
    return summary


if __name__ == '__main__':
    main(sys.argv[1:])
