"""CPU restatement of the langevinfts chain-propagator path (test oracle).

ORACLE / TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this file;
only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as
the checker.  Parity pinned: oracle/Makefile builds the reference CPU platform
itself (oracle/_ref), which passes all 27 reference golden tests, and
tests/test_oracle.py checks this restatement against that build and against
the golden vectors in tests/golden/.

Every function cites the reference code it restates (paths inside the
Langevin_FTS project).  numpy's FFT stands in for MKL DFTI; the conventions
(unnormalised forward r2c, backward normalised by 1/M, conjugate-even half
spectrum on the last axis) follow src/platforms/cpu/MklFFT3D.cpp:55-79.
"""
import numpy as np


# ---------------------------------------------------------------- tables
def padded3(nx, lx):
    """1D/2D boxes as 3D with leading 1s (src/common/Pseudo.cpp:25-40)."""
    dim = len(nx)
    tnx = [1] * (3 - dim) + list(nx)
    tdx = [1.0] * (3 - dim) + [lx[d] / nx[d] for d in range(dim)]
    return tnx, tdx


def boltz_bond(nx, lx, bond_length_sq, ds):
    """exp(-b^2 |k|^2 ds / 6) on the half spectrum (src/common/Pseudo.cpp:17-82)."""
    tnx, tdx = padded3(nx, lx)
    xf = [-bond_length_sq * (2 * np.pi / (tnx[d] * tdx[d])) ** 2 * ds / 6.0 for d in range(3)]
    i = np.arange(tnx[0]); i = np.where(i > tnx[0] // 2, tnx[0] - i, i)
    j = np.arange(tnx[1]); j = np.where(j > tnx[1] // 2, tnx[1] - j, j)
    k = np.arange(tnx[2] // 2 + 1)
    e = (i[:, None, None] ** 2 * xf[0] + j[None, :, None] ** 2 * xf[1] + k[None, None, :] ** 2 * xf[2])
    return np.exp(e)


def fourier_basis(nx, lx):
    """Weighted Fourier basis for stress (src/common/Pseudo.cpp:84-153); returns [3, ...]."""
    tnx, tdx = padded3(nx, lx)
    xf = [(2 * np.pi / (tnx[d] * tdx[d])) ** 2 for d in range(3)]
    i = np.arange(tnx[0]); i = np.where(i > tnx[0] // 2, tnx[0] - i, i)
    j = np.arange(tnx[1]); j = np.where(j > tnx[1] // 2, tnx[1] - j, j)
    k = np.arange(tnx[2] // 2 + 1)
    shape = (tnx[0], tnx[1], tnx[2] // 2 + 1)
    bx = np.broadcast_to(i[:, None, None] ** 2 * xf[0], shape).astype(float)
    by = np.broadcast_to(j[None, :, None] ** 2 * xf[1], shape).astype(float)
    bz = np.broadcast_to(k[None, None, :] ** 2 * xf[2], shape).astype(float)
    w = np.where((k != 0) & (2 * k != tnx[2]), 2.0, 1.0)[None, None, :]
    return np.stack([bx * w, by * w, bz * w])


def simpson_coeff(N):
    """Simpson 1/3 with 3/8 tail / trapezoid weights (src/common/SimpsonRule.h:10-59)."""
    if N == 0:
        return np.array([1.0])
    if N == 1:
        return np.array([0.5, 0.5])
    if N == 3:
        return np.array([3 / 8, 9 / 8, 9 / 8, 3 / 8])
    c = np.zeros(N + 1)
    if N % 2 == 0:
        c[0] = c[N] = 1 / 3
        c[1:N] = np.where(np.arange(1, N) % 2 == 1, 4 / 3, 2 / 3)
    else:
        c[0] = 1 / 3
        c[1:N - 3] = np.where(np.arange(1, N - 3) % 2 == 1, 4 / 3, 2 / 3)
        c[N - 3] = 3 / 8 + 1 / 3
        c[N - 2] = 9 / 8
        c[N - 1] = 9 / 8
        c[N] = 3 / 8
    return c


# ---------------------------------------------------------------- one step
class Grid:
    def __init__(self, nx, lx):
        self.nx = list(nx)
        self.lx = list(lx)
        self.tnx, self.tdx = padded3(nx, lx)
        self.M = int(np.prod(nx))
        self.shape = tuple(self.tnx)

    def fwd(self, q):
        return np.fft.rfftn(np.reshape(q, self.shape))

    def bwd(self, k):
        return np.fft.irfftn(k, s=self.shape, axes=(0, 1, 2)).reshape(-1)


def step_continuous(g, q_in, exp_dw, exp_dw_half, bond, bond_half):
    """4th-order Richardson step (src/platforms/cpu/CpuSolverPseudo.cpp:120-188)."""
    q1 = g.bwd(g.fwd(exp_dw * q_in) * bond) * exp_dw
    q2 = g.bwd(g.fwd(exp_dw_half * q_in) * bond_half) * exp_dw
    q2 = g.bwd(g.fwd(q2) * bond_half) * exp_dw_half
    return (4.0 * q2 - q1) / 3.0


def step_discrete(g, q_in, exp_dw, bond):
    """Bond-function step (src/platforms/cpu/CpuSolverPseudo.cpp:189-223)."""
    return g.bwd(g.fwd(q_in) * bond) * exp_dw


def half_bond_step(g, q_in, bond_half):
    """Half-bond step (src/platforms/cpu/CpuSolverPseudo.cpp:225-248)."""
    return g.bwd(g.fwd(q_in) * bond_half)


def segment_stress(g, q1, q2, bond_length_sq, basis, bond=None):
    """Single-segment stress sum (src/platforms/cpu/CpuSolverPseudo.cpp:250-356).
    Returns the 3 padded-3D components; DIM-D boxes use the last DIM."""
    k1, k2 = g.fwd(q1), g.fwd(q2)
    coeff = bond_length_sq * np.real(k1 * np.conj(k2))
    if bond is not None:
        coeff = coeff * bond
    return np.array([np.sum(coeff * basis[d]) for d in range(3)])


# ---------------------------------------------------------------- full solver
# ---------------------------------------------------------------- real-space step
BC_CODES = {"periodic": 0, "reflecting": 1, "absorbing": 2}


def laplacian_rows(n, dx, bond_length_sq, ds, bc_lo, bc_hi):
    """Tridiagonal rows (l, d, h) of one axis of the Crank-Nicolson step
    (src/common/FiniteDifference.cpp:20-99): off-diagonals -b^2 ds / (12 dx^2),
    diagonal 1 + b^2 ds / (6 dx^2); a reflecting side folds its outer
    off-diagonal into the diagonal, an absorbing side drops it."""
    xf = bond_length_sq * ds / (dx ** 2 * 6.0)
    l, d, h = np.full(n, -0.5 * xf), np.full(n, 1.0 + xf), np.full(n, -0.5 * xf)
    if bc_lo == 1:
        d[0] += l[0]; l[0] = 0.0
    elif bc_lo == 2:
        l[0] = 0.0
    if bc_hi == 1:
        d[-1] += h[-1]; h[-1] = 0.0
    elif bc_hi == 2:
        h[-1] = 0.0
    return l, d, h


def tridiagonal_lines(l, d, h, rhs, periodic):
    """Solve the tridiagonal (or cyclic, by Sherman-Morrison with gamma = 1)
    system along axis 0 of rhs for every other index at once
    (src/platforms/cpu/CpuSolverReal.cpp:480-549, same recurrences)."""
    n = rhs.shape[0]
    x = np.empty_like(rhs)
    c = np.zeros(n)
    if not periodic:
        t = d[0]
        x[0] = rhs[0] / t
        for i in range(1, n):
            c[i - 1] = h[i - 1] / t
            t = d[i] - l[i] * c[i - 1]
            x[i] = (rhs[i] - l[i] * x[i - 1]) / t
        for i in range(n - 2, -1, -1):
            x[i] = x[i] - c[i] * x[i + 1]
        return x
    q = np.zeros(n)
    t = d[0] - 1.0
    x[0] = rhs[0] / t
    q[0] = 1.0 / t
    for i in range(1, n - 1):
        c[i - 1] = h[i - 1] / t
        t = d[i] - l[i] * c[i - 1]
        x[i] = (rhs[i] - l[i] * x[i - 1]) / t
        q[i] = (-l[i] * q[i - 1]) / t
    c[n - 2] = h[n - 2] / t
    t = d[n - 1] - h[n - 1] * l[0] - l[n - 1] * c[n - 2]
    x[n - 1] = (rhs[n - 1] - l[n - 1] * x[n - 2]) / t
    q[n - 1] = (h[n - 1] - l[n - 1] * q[n - 2]) / t
    for i in range(n - 2, -1, -1):
        x[i] = x[i] - c[i] * x[i + 1]
        q[i] = q[i] - c[i] * q[i + 1]
    value = (x[0] + l[0] * x[n - 1]) / (1.0 + q[0] + l[0] * q[n - 1])
    return x - q.reshape([n] + [1] * (rhs.ndim - 1)) * value


def step_realspace(nx, lx, q_in, exp_dw, bond_length_sq, ds, bc):
    """One real-space Crank-Nicolson step, q_out = e ADI(e q_in), e = exp(-w ds/2)
    (src/platforms/cpu/CpuSolverReal.cpp:135-478): the first sweep implicit in
    axis 0 with the full explicit operator on the right, then one implicit
    sweep per further axis.  nx, lx: the box (1..3 axes); bc: 2 * dim names."""
    dim = len(nx)
    codes = [BC_CODES[b.lower()] for b in bc] if bc else [0] * (2 * dim)
    rows = [laplacian_rows(nx[a], lx[a] / nx[a], bond_length_sq, ds, codes[2 * a], codes[2 * a + 1]) for a in range(dim)]
    per = [codes[2 * a] == 0 for a in range(dim)]
    q = (exp_dw * q_in).reshape(nx)

    def shift(a, s_):  # q at i - 1 (s_ = -1) or i + 1 (s_ = +1) along axis a, with the boundary rule
        if per[a]:
            return np.roll(q, -s_, axis=a)
        idx = np.clip(np.arange(nx[a]) + s_, 0, nx[a] - 1)
        return np.take(q, idx, axis=a)

    def coef(a, r):  # row r of axis a broadcast along that axis
        shape = [1] * dim
        shape[a] = nx[a]
        return rows[a][r].reshape(shape)
    L, D, H = 0, 1, 2
    if dim == 1:
        rhs = (2.0 - coef(0, D)) * q - coef(0, L) * shift(0, -1) - coef(0, H) * shift(0, +1)
    else:
        inner = (float(dim) - 0.5 * coef(0, D) - sum(coef(a, D) for a in range(1, dim))) * q
        for a in range(dim - 1, 0, -1):
            inner = inner - coef(a, L) * shift(a, -1) - coef(a, H) * shift(a, +1)
        rhs = 2.0 * inner - coef(0, L) * shift(0, -1) - coef(0, H) * shift(0, +1)
    x = tridiagonal_lines(*rows[0], rhs, per[0])
    for a in range(1, dim):
        r = x + (coef(a, D) - 1.0) * q + coef(a, L) * shift(a, -1) + coef(a, H) * shift(a, +1)
        x = np.moveaxis(tridiagonal_lines(*rows[a], np.moveaxis(r, a, 0), per[a]), 0, a)
    return (x.reshape(-1) * exp_dw)


class PropagatorSolver:
    """compute_propagators / compute_concentrations / compute_stress for an
    arbitrary acyclic molecule, driven by the analyzer tables (propagators and
    blocks, e.g. from oracle/_ref/ref_schedule_dump).  Propagators are
    evaluated in height order; each one is independent of the stream schedule
    (src/platforms/cpu/CpuComputationContinuous.cpp:148-369, 371-465, 643-726;
    CpuComputationDiscrete.cpp:192-582, 584-679, 857-996)."""

    def __init__(self, nx, lx, model, ds, bond_lengths, polymers, analyzer):
        self.g = Grid(nx, lx)
        self.model = model
        self.ds = ds
        self.bond_lengths = dict(bond_lengths)
        self.polymers = polymers            # list of (volume_fraction, alpha)
        self.props = {p["key"]: p for p in analyzer["propagators"]}
        self.order = [p["key"] for p in analyzer["propagators"]]   # map order = height order
        self.blocks = analyzer["blocks"]
        self.update_laplacian_operator()

    def update_laplacian_operator(self):
        g = self.g
        self.bond = {m: boltz_bond(g.nx, g.lx, b * b, self.ds) for m, b in self.bond_lengths.items()}
        self.bond_half = {m: boltz_bond(g.nx, g.lx, b * b / 2, self.ds) for m, b in self.bond_lengths.items()}
        self.basis = fourier_basis(g.nx, g.lx)

    def set_lx(self, lx):
        self.g = Grid(self.g.nx, lx)
        self.update_laplacian_operator()

    def volume(self):
        return float(np.prod(self.g.lx))

    def compute_propagators(self, w):
        g, ds = self.g, self.ds
        M = g.M
        if self.model == "continuous":
            self.exp_dw = {m: np.exp(-w[m] * ds * 0.5) for m in w}
            self.exp_dw_half = {m: np.exp(-w[m] * ds * 0.25) for m in w}
        else:
            self.exp_dw = {m: np.exp(-w[m] * ds) for m in w}
        q, half = {}, {}
        for key in self.order:
            p = self.props[key]
            mt, N, deps = p["monomer_type"], p["max_n_segment"], p["deps"]
            e = self.exp_dw[mt]
            arr = np.zeros((N + 1, M))
            if self.model == "continuous":
                if not deps:
                    arr[0] = 1.0
                elif key[0] == "[":
                    arr[0] = sum(q[d][n] * r for d, n, r in deps)
                else:
                    arr[0] = np.prod([q[d][n] for d, n, r in deps], axis=0)
                for n in range(N):
                    arr[n + 1] = step_continuous(g, arr[n], e, self.exp_dw_half[mt], self.bond[mt], self.bond_half[mt])
                q[key] = arr
            else:
                hs = {}
                start = 1
                if not deps:
                    if N >= 1:
                        arr[1] = e
                elif key[0] == "[":
                    s = np.zeros(M)
                    for d, n, r in deps:
                        s += (half[d][0] if n == 0 else q[d][n]) * r
                    if deps[0][1] == 0:
                        hs[0] = s.copy()
                        arr[1] = half_bond_step(g, s, self.bond_half[mt]) * e
                    else:
                        arr[1] = step_discrete(g, s, e, self.bond[mt])
                else:
                    j = np.ones(M)
                    for d, n, r in deps:
                        j = j * half[d][n]
                    hs[0] = j
                    if N > 0:
                        arr[1] = half_bond_step(g, j, self.bond_half[mt]) * e
                if N >= 1:
                    if 1 in p["junction_ends"]:
                        hs[1] = half_bond_step(g, arr[1], self.bond_half[mt])
                    for n in range(start, N):
                        arr[n + 1] = step_discrete(g, arr[n], e, self.bond[mt])
                    for n in range(start, N):
                        if (n + 1) in p["junction_ends"]:
                            hs[n + 1] = half_bond_step(g, arr[n + 1], self.bond_half[mt])
                q[key] = arr
                half[key] = hs
        self.q, self.half = q, half
        # single-chain partition functions from the first block of each polymer
        dv = self.volume() / M
        self.Q = {}
        for b in self.blocks:
            p = b["polymer"]
            if p in self.Q:
                continue
            n_agg = len(b["v_u"]) // b["n_repeated"]
            NL = b["n_segment_left"]
            if self.model == "continuous":
                val = np.sum(dv * q[b["key_left"]][NL] * q[b["key_right"]][0])
            else:
                if NL == 0:
                    continue
                val = np.sum(dv * q[b["key_left"]][NL] * q[b["key_right"]][1] / self.exp_dw[b["monomer_type"]])
            self.Q[p] = val / n_agg / self.volume()

    def compute_concentrations(self):
        self.phi_block = {}
        for b in self.blocks:
            key = (b["polymer"], b["key_left"], b["key_right"])
            NR, NL = b["n_segment_right"], b["n_segment_left"]
            if NR == 0:
                self.phi_block[key] = np.zeros(self.g.M)
                continue
            q1, q2 = self.q[b["key_left"]], self.q[b["key_right"]]
            if self.model == "continuous":
                c = simpson_coeff(NR)
                phi = sum(c[n] * q1[NL - n] * q2[n] for n in range(NR + 1))
            else:
                phi = sum(q1[NL - n + 1] * q2[n] for n in range(1, NR + 1)) / self.exp_dw[b["monomer_type"]]
            vf, alpha = self.polymers[b["polymer"]]
            self.phi_block[key] = phi * (self.ds * vf / alpha / self.Q[b["polymer"]] * b["n_repeated"])

    def get_total_concentration(self, monomer_type):
        tot = np.zeros(self.g.M)
        for b in self.blocks:
            if b["monomer_type"] == monomer_type and b["n_segment_right"] != 0:
                tot += self.phi_block[(b["polymer"], b["key_left"], b["key_right"])]
        return tot

    def compute_stress(self):
        g = self.g
        dq = {}
        for b in self.blocks:
            p = b["polymer"]
            NR, NL, mt, rep = b["n_segment_right"], b["n_segment_left"], b["monomer_type"], b["n_repeated"]
            if NR == 0:
                continue
            q1, q2 = self.q[b["key_left"]], self.q[b["key_right"]]
            b2 = self.bond_lengths[mt] ** 2
            acc = np.zeros(3)
            if self.model == "continuous":
                c = simpson_coeff(NR)
                for n in range(NR + 1):
                    acc += segment_stress(g, q1[NL - n], q2[n], b2, self.basis) * c[n] * rep
            else:
                for n in range(NR + 1):
                    if n == NL:
                        if not self.props[b["key_left"]]["deps"]:
                            continue
                        s = segment_stress(g, self.half[b["key_left"]][0], q2[NR], b2 / 2, self.basis, self.bond_half[mt])
                    elif n == 0 and NL == NR:
                        if not self.props[b["key_right"]]["deps"]:
                            continue
                        s = segment_stress(g, q1[NL], self.half[b["key_right"]][0], b2 / 2, self.basis, self.bond_half[mt])
                    elif n == 0:
                        continue
                    else:
                        s = segment_stress(g, q1[NL - n], q2[n], b2, self.basis, self.bond[mt])
                    acc += s * rep
            dq[p] = dq.get(p, np.zeros(3)) + acc
        dim = len(g.nx)
        stress = np.zeros(dim)
        for p, (vf, alpha) in enumerate(self.polymers):
            d3 = dq.get(p, np.zeros(3))
            for d in range(dim):
                val = d3[3 - dim + d] / (-3.0 * g.lx[d] * g.M * g.M / self.ds)
                stress[d] += val * vf / alpha / self.Q[p]
        return stress


# ---------------------------------------------------------------- Anderson mixing
def find_an(u, v, n):
    """Gaussian elimination without pivoting (src/common/AndersonMixing.cpp:19-47)."""
    u = [list(r) for r in u]
    v = list(v)
    a = [0.0] * n
    for i in range(n):
        for j in range(i + 1, n):
            factor = u[j][i] / u[i][i]
            v[j] = v[j] - v[i] * factor
            for k in range(i + 1, n):
                u[j][k] = u[j][k] - u[i][k] * factor
    a[n - 1] = v[n - 1] / u[n - 1][n - 1]
    for i in range(n - 2, -1, -1):
        s = 0.0
        for j in range(i + 1, n):
            s = s + u[i][j] * a[j]
        a[i] = (v[i] - s) / u[i][i]
    return a


class AndersonMixing:
    """src/platforms/cpu/CpuAndersonMixing.cpp:76-161 with its circular buffers."""

    def __init__(self, n_var, max_hist, start_error, mix_min, mix_init):
        self.n_var, self.max_hist = n_var, max_hist
        self.start_error, self.mix_min, self.mix_init = start_error, mix_min, mix_init
        self.reset_count()

    def reset_count(self):
        self.mix = self.mix_init
        self.n_anderson = -1
        self.w_hist, self.d_hist, self.dots = [], [], []   # newest first

    def calculate_new_fields(self, w_current, w_deriv, old_error_level, error_level):
        if error_level < self.start_error or self.n_anderson >= 0:
            self.n_anderson += 1
        if self.n_anderson >= 0:
            self.n_anderson = min(self.max_hist, self.n_anderson)
            self.w_hist.insert(0, np.array(w_current, dtype=float))
            self.d_hist.insert(0, np.array(w_deriv, dtype=float))
            del self.w_hist[self.max_hist + 1:], self.d_hist[self.max_hist + 1:]
            row = [float(np.dot(w_deriv, self.d_hist[i])) for i in range(self.n_anderson + 1)]
            self.dots.insert(0, row)
            del self.dots[self.max_hist + 1:]
        if self.n_anderson <= 0:
            if old_error_level < error_level:
                self.mix = max(self.mix * 0.7, self.mix_min)
            else:
                self.mix = self.mix * 1.01
            return w_current + self.mix * w_deriv
        n = self.n_anderson
        d = self.dots
        v = [d[0][0] - d[0][i + 1] for i in range(n)]
        u = [[d[0][0] - d[0][i + 1] - d[0][j + 1] + d[min(i + 1, j + 1)][abs(i - j)] for j in range(n)] for i in range(n)]
        a = find_an(u, v, n)
        w1, d1 = self.w_hist[0], self.d_hist[0]
        w_new = w1 + d1
        for i in range(n):
            w_new = w_new + a[i] * (self.w_hist[i + 1] + self.d_hist[i + 1] - w1 - d1)
        return w_new
