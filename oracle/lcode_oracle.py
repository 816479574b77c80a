"""CPU oracle for the LCODE 3D xi-step: a numpy restatement of ``lcode.py``.

TEST INFRASTRUCTURE ONLY. This module is the checker for the CUDA product
path; it is imported by ``tests/``, by ``__graft_entry__.smoke()`` and by
``bench.py`` (its CPU-baseline sample and its ``--impl reference`` arm) and by
nothing else. The product package never imports it and never falls back to it.

Every function restates one function of the reference ``lcode.py`` (cited by
file:line) with the same argument meaning, in vectorised numpy:

* the particle kernels (``move_smart_kernel``, ``deposit_kernel``) become
  whole-array expressions; the deposition is a single ``np.bincount`` over
  the 9 stencil entries of every fine particle laid out particle-major in the
  reference's stencil order, which accumulates each cell in exactly the order
  a serial loop over fine particles does (the reference's GPU order is
  arbitrary, its float64 atomics make it non-deterministic);
* the padded-rFFT DST-I / DCT-I constructions (``dst2d``, ``mix2d``,
  ``dct2d``) are replaced by the transforms they realise, computed with
  ``scipy.fft`` (pocketfft): ``dst2d == dstn(type=1)``,
  ``dct2d == -dctn(type=1)``, ``mix2d`` = zero-bordered DST-I(axis 0) x
  DCT-I(axis 1). The equalities are checked against the reference's own
  outputs in ``tests/test_oracle.py``.

Parity of this oracle is pinned against golden vectors produced by the
reference itself (``tests/golden/make_golden.py``).
"""
import functools
import math
import types

import numpy as np
import scipy.fft

ELECTRON_CHARGE = -1   # lcode.py:46
ELECTRON_MASS = 1      # lcode.py:47

# threads used by scipy.fft; bench.py raises it for the multi-core baseline
FFT_WORKERS = 1


# ---------------------------------------------------------------------------
# Spectral transforms (lcode.py:124-141, 190-212, 295-313)
# ---------------------------------------------------------------------------

def dst2d(a):
    """DST-I along both axes, unnormalised (lcode.py:124-141)."""
    assert a.shape[0] == a.shape[1]
    return scipy.fft.dstn(a, type=1, workers=FFT_WORKERS)


def mix2d(a):
    """DST-I along axis 0 then DCT-I along axis 1; output has one zero row
    added above and below (lcode.py:190-212)."""
    M, N = a.shape
    out = np.zeros((M + 2, N))
    t = scipy.fft.dst(a, type=1, axis=0, workers=FFT_WORKERS)
    out[1:M + 1] = scipy.fft.dct(t, type=1, axis=1, workers=FFT_WORKERS)
    return out


def dct2d(a):
    """Minus the DCT-I along both axes, unnormalised (lcode.py:295-313)."""
    assert a.shape[0] == a.shape[1]
    return -scipy.fft.dctn(a, type=1, workers=FFT_WORKERS)


def _lam(k, grid_steps, grid_step_size):
    # lam[k] = 4 / h**2 * sin(k * pi / (2 (N - 1)))**2  (lcode.py:152-154)
    return 4 / grid_step_size ** 2 * np.sin(k * np.pi / (2 * (grid_steps - 1))) ** 2


@functools.lru_cache(maxsize=None)
def dirichlet_matrix(grid_steps, grid_step_size):
    """1 / (lam_i + lam_j) / (2 (N - 1))**2, k = 1..N-2 (lcode.py:144-157)."""
    lam = _lam(np.arange(1, grid_steps - 1), grid_steps, grid_step_size)
    mul = 1 / (lam[:, None] + lam[None, :])
    return mul / (2 * (grid_steps - 1)) ** 2


@functools.lru_cache(maxsize=None)
def mixed_matrix(grid_steps, grid_step_size, subtraction_trick):
    """1 / (lam_i + lam_j (+1)) / (2 (N - 1))**2 with i = 1..N-2 and
    j = 0..N-1 (lcode.py:215-231)."""
    li = _lam(np.arange(1, grid_steps - 1), grid_steps, grid_step_size)
    lj = _lam(np.arange(grid_steps), grid_steps, grid_step_size)
    mul = 1 / (li[:, None] + lj[None, :] + (1 if subtraction_trick else 0))
    return mul / (2 * (grid_steps - 1)) ** 2


@functools.lru_cache(maxsize=None)
def neumann_matrix(grid_steps, grid_step_size):
    """1 / (lam_i + lam_j), k = 0..N-1, with the [0, 0] entry set to 0
    (lcode.py:316-330)."""
    lam = _lam(np.arange(grid_steps), grid_steps, grid_step_size)
    with np.errstate(divide='ignore'):
        mul = 1 / (lam[:, None] + lam[None, :])
    mul[0, 0] = 0
    return mul / (2 * (grid_steps - 1)) ** 2


# ---------------------------------------------------------------------------
# Field solvers (lcode.py:160-184, 234-290, 333-364)
# ---------------------------------------------------------------------------

def calculate_Ez(config, jx, jy):
    """Dirichlet Poisson solve for Ez (lcode.py:160-184)."""
    h = config.grid_step_size
    djx_dx = jx[2:, 1:-1] - jx[:-2, 1:-1]
    djy_dy = jy[1:-1, 2:] - jy[1:-1, :-2]
    rhs_inner = -(djx_dx + djy_dy) / (h * 2)
    f = dst2d(rhs_inner)
    f *= dirichlet_matrix(config.grid_steps, h)
    Ez_inner = dst2d(f)
    return np.pad(Ez_inner, 1, 'constant', constant_values=0)


def dx_dy(arr, grid_step_size):
    """Centred x and y differences, zero border (lcode.py:234-243)."""
    dx, dy = np.zeros_like(arr), np.zeros_like(arr)
    dx[1:-1, 1:-1] = arr[2:, 1:-1] - arr[:-2, 1:-1]
    dy[1:-1, 1:-1] = arr[1:-1, 2:] - arr[1:-1, :-2]
    return dx / (grid_step_size * 2), dy / (grid_step_size * 2)


def calculate_Ex_Ey_Bx_By(config, Ex_avg, Ey_avg, Bx_avg, By_avg,
                          beam_ro, ro, jx, jy, jz, jx_prev, jy_prev):
    """Helmholtz/Laplace solves with mixed boundary conditions for the
    transverse fields; Ex and By are solved transposed (lcode.py:246-290)."""
    h = config.grid_step_size
    dro_dx, dro_dy = dx_dy(ro + beam_ro, h)
    djz_dx, djz_dy = dx_dy(jz + beam_ro, h)
    djx_dxi = (jx_prev - jx) / config.xi_step_size
    djy_dxi = (jy_prev - jy) / config.xi_step_size
    st = config.field_solver_subtraction_trick
    Ex_rhs = -((dro_dx - djx_dxi) - Ex_avg * st)
    Ey_rhs = -((dro_dy - djy_dxi) - Ey_avg * st)
    Bx_rhs = +((djz_dy - djy_dxi) + Bx_avg * st)
    By_rhs = -((djz_dx - djx_dxi) - By_avg * st)
    mix_mat = mixed_matrix(config.grid_steps, h, st)
    Ey = mix2d(mix_mat * mix2d(Ey_rhs[1:-1, :])[1:-1, :])
    Bx = mix2d(mix_mat * mix2d(Bx_rhs[1:-1, :])[1:-1, :])
    By = mix2d(mix_mat * mix2d(By_rhs.T[1:-1, :])[1:-1, :]).T
    Ex = mix2d(mix_mat * mix2d(Ex_rhs.T[1:-1, :])[1:-1, :]).T
    return Ex, Ey, Bx, By


def calculate_Bz(config, jx, jy):
    """Neumann Poisson solve for Bz, then mean subtraction
    (lcode.py:333-364)."""
    h = config.grid_step_size
    djx_dy = jx[1:-1, 2:] - jx[1:-1, :-2]
    djy_dx = jy[2:, 1:-1] - jy[:-2, 1:-1]
    djx_dy = np.pad(djx_dy, 1, 'constant', constant_values=0)
    djy_dx = np.pad(djy_dx, 1, 'constant', constant_values=0)
    rhs = -(djx_dy - djy_dx) / (h * 2)
    f = dct2d(rhs)
    f *= neumann_matrix(config.grid_steps, h)
    Bz = dct2d(f)
    Bz -= Bz.mean()
    return Bz


# ---------------------------------------------------------------------------
# Particles: TSC weights, pusher, deposition (lcode.py:369-449, 576-823)
# ---------------------------------------------------------------------------

def weights(x, y, grid_steps, grid_step_size):
    """Cell indices and the 9 TSC weights, in the reference's order
    MP, 0P, PP, M0, 00, P0, MM, 0M, PM (lcode.py:396-418)."""
    x_h, y_h = x / grid_step_size + .5, y / grid_step_size + .5
    fx, fy = np.floor(x_h), np.floor(y_h)
    i = fx.astype(np.int64) + grid_steps // 2
    j = fy.astype(np.int64) + grid_steps // 2
    x_loc, y_loc = x_h - fx - .5, y_h - fy - .5
    wx0, wy0 = .75 - x_loc ** 2, .75 - y_loc ** 2
    wxP, wyP = (.5 + x_loc) ** 2 / 2, (.5 + y_loc) ** 2 / 2
    wxM, wyM = (.5 - x_loc) ** 2 / 2, (.5 - y_loc) ** 2 / 2
    w = (wxM * wyP, wx0 * wyP, wxP * wyP,
         wxM * wy0, wx0 * wy0, wxP * wy0,
         wxM * wyM, wx0 * wyM, wxP * wyM)
    return i, j, w


# (di, dj) offsets in the same order as the weights (lcode.py:427-429, 441-449)
STENCIL = ((-1, +1), (0, +1), (+1, +1),
           (-1, 0), (0, 0), (+1, 0),
           (-1, -1), (0, -1), (+1, -1))


def _check_stencil(i, j, N):
    if i.size and (i.min() < 1 or i.max() > N - 2 or j.min() < 1 or j.max() > N - 2):
        raise IndexError('particle stencil leaves the grid: a particle '
                         'reached the outermost cells')


def interp9(a, i, j, w):
    """Weighted 3x3 gather (lcode.py:421-430)."""
    s = 0.
    for (di, dj), wk in zip(STENCIL, w):
        s = s + a[i + di, j + dj] * wk
    return s


def move_estimate_wo_fields(config, m, x_init, y_init, prev_x_offt,
                            prev_y_offt, px, py, pz):
    """Field-free drift with coordinate reflection at +-reflect_boundary
    using >= / <= (lcode.py:369-391)."""
    x, y = x_init + prev_x_offt, y_init + prev_y_offt
    gamma_m = np.sqrt(m ** 2 + pz ** 2 + px ** 2 + py ** 2)
    x = x + px / (gamma_m - pz) * config.xi_step_size
    y = y + py / (gamma_m - pz) * config.xi_step_size
    r = config.reflect_boundary
    for a in (x, y):
        s = a >= +r
        a[s] = +2 * r - a[s]
        s = a <= -r
        a[s] = -2 * r - a[s]
    return x - x_init, y - y_init


def move_smart(config, m, q, x_init, y_init, x_prev_offt, y_prev_offt,
               estimated_x_offt, estimated_y_offt, px_prev, py_prev, pz_prev,
               Ex_avg, Ey_avg, Ez_avg, Bx_avg, By_avg, Bz_avg):
    """Half-step field gather, two-pass momentum predictor, position update
    and reflection of position and momentum with > / < (lcode.py:704-823)."""
    shape = np.shape(x_prev_offt)
    f = lambda a: np.ascontiguousarray(np.broadcast_to(a, shape), dtype=np.float64).ravel()
    m, q, x_init, y_init = f(m), f(q), f(x_init), f(y_init)
    x_offt, y_offt = f(x_prev_offt).copy(), f(y_prev_offt).copy()
    ex, ey = f(estimated_x_offt), f(estimated_y_offt)
    opx, opy, opz = f(px_prev), f(py_prev), f(pz_prev)
    dxi = config.xi_step_size
    N = config.grid_steps

    x_half = x_init + (x_offt + ex) / 2
    y_half = y_init + (y_offt + ey) / 2
    i, j, w = weights(x_half, y_half, N, config.grid_step_size)
    _check_stencil(i, j, N)
    Ex = interp9(Ex_avg, i, j, w)
    Ey = interp9(Ey_avg, i, j, w)
    Ez = interp9(Ez_avg, i, j, w)
    Bx = interp9(Bx_avg, i, j, w)
    By = interp9(By_avg, i, j, w)
    Bz = interp9(Bz_avg, i, j, w)

    px, py, pz = opx, opy, opz
    for _ in range(2):
        gamma_m = np.sqrt(m ** 2 + pz ** 2 + px ** 2 + py ** 2)
        vx, vy, vz = px / gamma_m, py / gamma_m, pz / gamma_m
        factor_1 = q * dxi / (1 - pz / gamma_m)
        dpx = factor_1 * (Ex + vy * Bz - vz * By)
        dpy = factor_1 * (Ey - vx * Bz + vz * Bx)
        dpz = factor_1 * (Ez + vx * By - vy * Bx)
        px, py, pz = opx + dpx / 2, opy + dpy / 2, opz + dpz / 2

    gamma_m = np.sqrt(m ** 2 + pz ** 2 + px ** 2 + py ** 2)
    x_offt = x_offt + px / (gamma_m - pz) * dxi
    y_offt = y_offt + py / (gamma_m - pz) * dxi
    px, py, pz = opx + dpx, opy + dpy, opz + dpz

    r = config.reflect_boundary
    x = x_init + x_offt
    y = y_init + y_offt
    for a, a_init, a_offt, p in ((x, x_init, x_offt, px), (y, y_init, y_offt, py)):
        s = a > +r
        a[s] = +2 * r - a[s]
        a_offt[s] = a[s] - a_init[s]
        p[s] = -p[s]
        s = a < -r
        a[s] = -2 * r - a[s]
        a_offt[s] = a[s] - a_init[s]
        p[s] = -p[s]
    return tuple(v.reshape(shape) for v in (x_offt, y_offt, px, py, pz))


def coarse_to_fine(c_x_offt, c_y_offt, c_m, c_q, c_px, c_py, c_pz,
                   virtplasma_smallness_factor, fine_grid,
                   influence_prev, influence_next, indices_prev, indices_next):
    """Bilinear coarse->fine interpolation of all fine particles, in (fi, fj)
    row-major order (lcode.py:576-621)."""
    ip, inn = influence_prev, influence_next
    A = ip[:, None] * ip[None, :]
    B = ip[:, None] * inn[None, :]
    C = inn[:, None] * ip[None, :]
    D = inn[:, None] * inn[None, :]
    pi, ni = indices_prev[:, None], indices_next[:, None]
    pj, nj = indices_prev[None, :], indices_next[None, :]

    def mix(c):
        return A * c[pi, pj] + B * c[pi, nj] + C * c[ni, pj] + D * c[ni, nj]
    x = fine_grid[:, None] + mix(c_x_offt)
    y = fine_grid[None, :] + mix(c_y_offt)
    s = virtplasma_smallness_factor
    return (x, y, s * mix(c_m), s * mix(c_q),
            s * mix(c_px), s * mix(c_py), s * mix(c_pz))


def deposit(config, ro_initial, x_offt, y_offt, m, q, px, py, pz, virt_params):
    """Coarse->fine interpolation and 9-point TSC deposition of rho, jx, jy,
    jz, then + ro_initial (lcode.py:626-689)."""
    N = config.grid_steps
    sf = 1 / (config.plasma_coarseness * config.plasma_fineness) ** 2
    v = virt_params
    x, y, mf, qf, pxf, pyf, pzf = coarse_to_fine(
        x_offt, y_offt, m, q, px, py, pz, sf, v.fine_grid,
        v.influence_prev, v.influence_next, v.indices_prev, v.indices_next)
    gamma_m = np.sqrt(mf ** 2 + pxf ** 2 + pyf ** 2 + pzf ** 2)
    dro = qf / (1 - pzf / gamma_m)
    djx = pxf * (dro / gamma_m)
    djy = pyf * (dro / gamma_m)
    djz = pzf * (dro / gamma_m)
    i, j, w = weights(x.ravel(), y.ravel(), N, config.grid_step_size)
    _check_stencil(i, j, N)
    idx = np.stack([(i + di) * N + (j + dj) for di, dj in STENCIL], axis=1).ravel()
    W = np.stack(w, axis=1)
    out = []
    for val in (dro, djx, djy, djz):
        contrib = (val.ravel()[:, None] * W).ravel()
        out.append(np.bincount(idx, weights=contrib, minlength=N * N).reshape(N, N))
    ro, jx, jy, jz = out
    ro = ro + ro_initial
    return ro, jx, jy, jz


# ---------------------------------------------------------------------------
# Plasma layout and init (lcode.py:454-573, 692-699, 936-975)
# ---------------------------------------------------------------------------

def make_coarse_plasma_grid(steps, step_size, coarseness=3):
    """Symmetric coarse lattice with spacing h*c (lcode.py:454-465)."""
    assert coarseness == int(coarseness)
    right = np.arange(steps // (coarseness * 2)) * (step_size * coarseness)
    return np.concatenate([-right[:0:-1], right])


def make_fine_plasma_grid(steps, step_size, fineness=2):
    """Symmetric fine lattice with spacing h/f, avoiding cell edges
    (lcode.py:468-487)."""
    assert fineness == int(fineness)
    step = step_size / fineness
    if fineness % 2:
        right = np.arange(steps // 2 * fineness) * step
        return np.concatenate([-right[:0:-1], right])
    right = (.5 + np.arange(steps // 2 * fineness)) * step
    return np.concatenate([-right[::-1], right])


def make_plasma(steps, cell_size, coarseness=3, fineness=2):
    """Coarse particle arrays and the coarse->fine interpolation parameters
    (lcode.py:490-573)."""
    coarse_step = cell_size * coarseness
    cg = make_coarse_plasma_grid(steps, cell_size, coarseness)
    fg = make_fine_plasma_grid(steps, cell_size, fineness)
    Nc = len(cg)
    x_init = np.broadcast_to(cg[:, None], (Nc, Nc)).copy()
    y_init = np.broadcast_to(cg[None, :], (Nc, Nc)).copy()
    z = lambda: np.zeros((Nc, Nc))
    m = np.ones((Nc, Nc)) * ELECTRON_MASS * coarseness ** 2
    q = np.ones((Nc, Nc)) * ELECTRON_CHARGE * coarseness ** 2
    idx = np.searchsorted(cg, fg)
    indices_next = np.clip(idx, 0, Nc - 1)
    indices_prev = np.clip(idx - 1, 0, Nc - 1)
    influence_prev = (cg[indices_next] - fg) / coarse_step
    influence_next = (fg - cg[indices_prev]) / coarse_step
    influence_prev[indices_next == 0] = 0
    influence_next[indices_next == 0] = 1
    influence_next[indices_prev == Nc - 1] = 0
    influence_prev[indices_prev == Nc - 1] = 1
    virt = types.SimpleNamespace(influence_prev=influence_prev,
                                 influence_next=influence_next,
                                 indices_prev=indices_prev,
                                 indices_next=indices_next, fine_grid=fg)
    return x_init, y_init, z(), z(), z(), z(), z(), m, q, virt


def init(config):
    """Validate the config, set reflect_boundary, build plasma and the ion
    background (lcode.py:936-975)."""
    assert config.grid_steps % 2 == 1
    assert config.reflect_padding_steps > config.plasma_coarseness + 1
    config.reflect_boundary = config.grid_step_size * (
        config.grid_steps / 2 - config.reflect_padding_steps)
    N = config.grid_steps
    grid = (np.arange(N) - N // 2) * config.grid_step_size
    xs, ys = grid[:, None], grid[None, :]
    x_init, y_init, x_offt, y_offt, px, py, pz, m, q, virt = make_plasma(
        N - config.plasma_padding_steps * 2, config.grid_step_size,
        coarseness=config.plasma_coarseness, fineness=config.plasma_fineness)
    ro_e, _, _, _ = deposit(config, 0, x_offt, y_offt, m, q, px, py, pz, virt)
    const = types.SimpleNamespace(m=m, q=q, x_init=x_init, y_init=y_init,
                                  ro_initial=-ro_e)
    z = lambda: np.zeros((N, N))
    state = types.SimpleNamespace(x_offt=x_offt, y_offt=y_offt, px=px, py=py,
                                  pz=pz, Ex=z(), Ey=z(), Ez=z(), Bx=z(),
                                  By=z(), Bz=z(), ro=z(), jx=z(), jy=z(), jz=z())
    return xs, ys, const, virt, state


# ---------------------------------------------------------------------------
# The xi step (lcode.py:828-931)
# ---------------------------------------------------------------------------

def _fields(config, prev, Ex_sub, Ey_sub, Bx_sub, By_sub, beam_ro, ro, jx, jy, jz):
    A = config.field_solver_variant_A
    ro_in = (ro + prev.ro) / 2 if A else ro
    jz_in = (jz + prev.jz) / 2 if A else jz
    Ex, Ey, Bx, By = calculate_Ex_Ey_Bx_By(config, Ex_sub, Ey_sub, Bx_sub,
                                           By_sub, beam_ro, ro_in, jx, jy,
                                           jz_in, prev.jx, prev.jy)
    if A:
        Ex, Ey = 2 * Ex - prev.Ex, 2 * Ey - prev.Ey
        Bx, By = 2 * Bx - prev.Bx, 2 * By - prev.By
    Ez = calculate_Ez(config, jx, jy)
    Bz = calculate_Bz(config, jx, jy)
    return Ex, Ey, Ez, Bx, By, Bz


def step(config, const, virt_params, prev, beam_ro):
    """Estimate, predictor (move/deposit/fields/average), corrector, final
    move/deposit; fields of the corrector, particles and densities of the
    final pass (lcode.py:828-931)."""
    beam_ro = np.broadcast_to(np.asarray(beam_ro, dtype=np.float64),
                              (config.grid_steps,) * 2)
    c = const
    x_offt, y_offt = move_estimate_wo_fields(config, c.m, c.x_init, c.y_init,
                                             prev.x_offt, prev.y_offt,
                                             prev.px, prev.py, prev.pz)
    avg = (prev.Ex, prev.Ey, prev.Ez, prev.Bx, prev.By, prev.Bz)
    sub = (prev.Ex, prev.Ey, prev.Bx, prev.By)
    for _ in range(2):
        x_offt, y_offt, px, py, pz = move_smart(
            config, c.m, c.q, c.x_init, c.y_init, prev.x_offt, prev.y_offt,
            x_offt, y_offt, prev.px, prev.py, prev.pz, *avg)
        ro, jx, jy, jz = deposit(config, c.ro_initial, x_offt, y_offt, c.m,
                                 c.q, px, py, pz, virt_params)
        Ex, Ey, Ez, Bx, By, Bz = _fields(config, prev, *sub, beam_ro,
                                         ro, jx, jy, jz)
        avg = tuple((F + Fp) / 2 for F, Fp in zip(
            (Ex, Ey, Ez, Bx, By, Bz),
            (prev.Ex, prev.Ey, prev.Ez, prev.Bx, prev.By, prev.Bz)))
        sub = (avg[0], avg[1], avg[3], avg[4])
    x_offt, y_offt, px, py, pz = move_smart(
        config, c.m, c.q, c.x_init, c.y_init, prev.x_offt, prev.y_offt,
        x_offt, y_offt, prev.px, prev.py, prev.pz, *avg)
    ro, jx, jy, jz = deposit(config, c.ro_initial, x_offt, y_offt, c.m, c.q,
                             px, py, pz, virt_params)
    return types.SimpleNamespace(x_offt=x_offt, y_offt=y_offt, px=px, py=py,
                                 pz=pz, Ex=Ex, Ey=Ey, Ez=Ez, Bx=Bx, By=By,
                                 Bz=Bz, ro=ro, jx=jx, jy=jy, jz=jz)


def diags_ro_zn_value(config, ro):
    """The noise figure of diags_ro_zn (lcode.py:979-987) for one array,
    without the running maximum: mean |ro - gaussian_filter(ro, 0.25 / h)|
    / 4.23045376e-04 (scipy.ndimage, the reference's own call)."""
    import scipy.ndimage
    ro = np.asarray(ro, dtype=np.float64)
    sigma = 0.25 / config.grid_step_size
    blurred = scipy.ndimage.gaussian_filter(ro, sigma=sigma)
    return float(np.abs(ro - blurred).mean() / 4.23045376e-04)


def relative_error(a, b):
    """max|a - b| / max|b|, the per-field parity measure."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    den = np.abs(b).max()
    num = np.abs(a - b).max()
    return num / den if den > 0 else num


# ---------------------------------------------------------------------------
# Optional C restatement of the two particle kernels (oracle/lc3d_oracle.c),
# bit-identical to the numpy forms above with one thread; used for speed at
# 641^2 and, multi-threaded, as bench.py's multi-core CPU baseline.
# ---------------------------------------------------------------------------

_C = None
_C_THREADS = 1


def use_c_kernels(nthreads=1):
    """Route move_smart / deposit through oracle/liblc3d_oracle.so."""
    global _C, _C_THREADS, move_smart, deposit
    import ctypes
    from . import build as _b
    lib = ctypes.CDLL(_b.build())
    P = ctypes.c_void_p
    lib.oracle_move_smart.restype = ctypes.c_int
    lib.oracle_move_smart.argtypes = [ctypes.c_int] + [P] * 17 + [ctypes.c_int, ctypes.c_double,
                                                               ctypes.c_double, ctypes.c_double] + [P] * 5 + [ctypes.c_int]
    lib.oracle_deposit.restype = ctypes.c_int
    lib.oracle_deposit.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 2 + [P] * 16 + [ctypes.c_int]
    _C, _C_THREADS = lib, max(1, int(nthreads))
    move_smart, deposit = _move_smart_c, _deposit_c


def use_numpy_kernels():
    global move_smart, deposit
    move_smart, deposit = _move_smart_np, _deposit_np


_move_smart_np, _deposit_np = move_smart, deposit


def _f(a, shape):
    return np.ascontiguousarray(np.broadcast_to(np.asarray(a, dtype=np.float64), shape))


def _p(a):
    return a.ctypes.data


def _move_smart_c(config, m, q, x_init, y_init, x_prev_offt, y_prev_offt,
                  estimated_x_offt, estimated_y_offt, px_prev, py_prev, pz_prev,
                  Ex_avg, Ey_avg, Ez_avg, Bx_avg, By_avg, Bz_avg):
    shape = np.shape(x_prev_offt)
    ins = [_f(a, shape) for a in (m, q, x_init, y_init, x_prev_offt, y_prev_offt,
                                  estimated_x_offt, estimated_y_offt, px_prev, py_prev, pz_prev)]
    N = config.grid_steps
    flds = [_f(a, (N, N)) for a in (Ex_avg, Ey_avg, Ez_avg, Bx_avg, By_avg, Bz_avg)]
    outs = [np.empty(shape) for _ in range(5)]
    bad = _C.oracle_move_smart(int(np.prod(shape)), *[_p(a) for a in ins + flds], N,
                               config.grid_step_size, config.xi_step_size,
                               config.reflect_boundary, *[_p(o) for o in outs], _C_THREADS)
    if bad:
        raise IndexError('particle stencil leaves the grid')
    return tuple(outs)


def _deposit_c(config, ro_initial, x_offt, y_offt, m, q, px, py, pz, virt_params):
    v = virt_params
    shape = np.shape(x_offt)
    ins = [_f(a, shape) for a in (x_offt, y_offt, m, q, px, py, pz)]
    vf = [np.ascontiguousarray(v.influence_prev, dtype=np.float64),
          np.ascontiguousarray(v.influence_next, dtype=np.float64),
          np.ascontiguousarray(v.indices_prev, dtype=np.int64),
          np.ascontiguousarray(v.indices_next, dtype=np.int64),
          np.ascontiguousarray(v.fine_grid, dtype=np.float64)]
    N = config.grid_steps
    out = [np.zeros((N, N)) for _ in range(4)]
    sf = 1 / (config.plasma_coarseness * config.plasma_fineness) ** 2
    bad = _C.oracle_deposit(shape[0], len(vf[4]), N, config.grid_step_size, sf,
                            *[_p(a) for a in ins + vf + out], _C_THREADS)
    if bad:
        raise IndexError('particle stencil leaves the grid')
    ro, jx, jy, jz = out
    return ro + ro_initial, jx, jy, jz
