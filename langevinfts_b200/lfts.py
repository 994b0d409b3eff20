"""Langevin field-theoretic simulation drivers.

`LFTS` runs one system through the public `langevinfts` API (numpy arrays in
and out, exactly the calls the reference driver examples/fts/lfts.py makes per
saddle-point iteration: compute_propagators, compute_concentrations,
get_total_concentration, AndersonMixing.calculate_new_fields).  It works with
this package's module or any module with the same API, so the same driver
times and checks both.  Plotting, .mat recording and the structure function
of the reference driver are left out; the step arithmetic is the same:
  SymmetricPolymerTheory           lfts.py:20-274
  Leimkuhler-Matthews update       lfts.py:697-706
  saddle point by Anderson mixing  lfts.py:807-868
  failed saddle point: restore     lfts.py:713-730

`BatchedLFTS` advances many independent replicas (one PCG64 stream each) on
the device-resident engine `langevinfts.BatchedLangevin`; replica r with seed
s_r follows the same trajectory as `LFTS(params, random_seed=s_r)`.
"""
import itertools
import re

import numpy as np


def calculate_sigma(langevin_nbar, langevin_dt, n_grids, volume):
    """Standard deviation of the Langevin noise (lfts.py:17-18)."""
    return np.sqrt(2 * langevin_dt * n_grids / (volume * np.sqrt(langevin_nbar)))


class SymmetricPolymerTheory:
    """Multi-monomer field theory with the symmetric choice of auxiliary fields
    (restates lfts.py:20-274: eigen-decomposition of the projected chi matrix,
    Hamiltonian coefficients and functional derivatives)."""

    def __init__(self, monomer_types, chi_n):
        self.monomer_types = monomer_types
        S = len(monomer_types)
        self.matrix_q = np.ones((S, S)) / S
        self.matrix_p = np.identity(S) - self.matrix_q
        eigenvalues, matrix_o = self.compute_eigen_system(chi_n, self.matrix_p)
        matrix_chi = np.zeros((S, S))
        for i in range(S):
            for j in range(i + 1, S):
                key = ",".join(sorted([monomer_types[i], monomer_types[j]]))
                if key in chi_n:
                    matrix_chi[i, j] = matrix_chi[j, i] = chi_n[key]
        self.matrix_chi = matrix_chi
        self.vector_s = matrix_chi @ np.ones(S) / S
        self.vector_large_s = matrix_o.T @ self.vector_s
        self.aux_fields_real_idx, self.aux_fields_imag_idx = [], []
        for i in range(S - 1):
            if np.isclose(eigenvalues[i], 0.0):
                print("One of eigenvalues is zero for given chiN values.")
            elif eigenvalues[i] > 0:
                self.aux_fields_imag_idx.append(i)
            else:
                self.aux_fields_real_idx.append(i)
        self.aux_fields_imag_idx.append(S - 1)
        self.R = len(self.aux_fields_real_idx)
        self.I = len(self.aux_fields_imag_idx)
        self.h_const, self.h_coef_mu1, self.h_coef_mu2 = self.compute_h_coef(chi_n, eigenvalues)
        self.matrix_a = matrix_o.copy()
        self.matrix_a_inv = matrix_o.T.copy() / S
        assert np.isclose(np.std(self.matrix_a @ self.matrix_a_inv - np.identity(S)), 0.0)
        eps = 1e-5
        self.h_const_deriv_chin, self.h_coef_mu1_deriv_chin, self.h_coef_mu2_deriv_chin = {}, {}, {}
        for key in chi_n:
            cp, cn = dict(chi_n), dict(chi_n)
            cp[key] += eps
            cn[key] -= eps
            ep, _ = self.compute_eigen_system(cp, self.matrix_p)
            en, _ = self.compute_eigen_system(cn, self.matrix_p)
            hp = self.compute_h_coef(cp, ep)
            hn = self.compute_h_coef(cn, en)
            self.h_const_deriv_chin[key] = (hp[0] - hn[0]) / (2 * eps)
            self.h_coef_mu1_deriv_chin[key] = (hp[1] - hn[1]) / (2 * eps)
            self.h_coef_mu2_deriv_chin[key] = (hp[2] - hn[2]) / (2 * eps)
        self.eigenvalues = eigenvalues
        self.matrix_o = matrix_o

    def to_aux_fields(self, w):
        return self.matrix_a_inv @ w

    def to_monomer_fields(self, w_aux):
        return self.matrix_a @ w_aux

    def compute_eigen_system(self, chi_n, matrix_p):
        S = matrix_p.shape[0]
        matrix_chi = np.zeros((S, S))
        for i in range(S):
            for j in range(i + 1, S):
                key = ",".join(sorted([self.monomer_types[i], self.monomer_types[j]]))
                if key in chi_n:
                    matrix_chi[i, j] = matrix_chi[j, i] = chi_n[key]
        eigenvalues, eigenvectors = np.linalg.eigh(matrix_p @ (matrix_chi @ matrix_p))
        order = np.argsort(np.abs(eigenvalues))[::-1]
        eigenvalues, eigenvectors = eigenvalues[order], eigenvectors[:, order]
        eigenvectors[:, -1] = np.ones(S) / np.sqrt(S)
        zero = np.isclose(eigenvalues, 0.0, atol=1e-12)
        eigenvalues[zero] = 0.0
        v0 = eigenvectors[:, zero]
        for i in range(v0.shape[1] - 2, -1, -1):
            base = v0[:, i].copy()
            for j in range(i + 1, v0.shape[1]):
                v0[:, i] -= v0[:, j] * np.dot(base, v0[:, j])
            v0[:, i] /= np.linalg.norm(v0[:, i])
        eigenvectors[:, zero] = v0
        for i in range(S):
            if eigenvectors[0, i] < 0.0:
                eigenvectors[:, i] *= -1.0
        return eigenvalues, eigenvectors * np.sqrt(S)

    def compute_h_coef(self, chi_n, eigenvalues):
        S = len(self.monomer_types)
        h_const = 0.5 * np.sum(self.vector_s) / S
        mu1, mu2 = np.zeros(S - 1), np.zeros(S - 1)
        for i in range(S - 1):
            if not np.isclose(eigenvalues[i], 0.0):
                h_const -= 0.5 * self.vector_large_s[i] ** 2 / eigenvalues[i] / S
                mu1[i] = self.vector_large_s[i] / eigenvalues[i]
                mu2[i] = -0.5 / eigenvalues[i] * S
        return h_const, mu1, mu2

    def compute_hamiltonian(self, molecules, w_aux, total_partitions):
        S = len(self.monomer_types)
        h = -np.mean(w_aux[S - 1])
        for i in range(S - 1):
            h += self.h_coef_mu2[i] * np.mean(w_aux[i] ** 2) + self.h_coef_mu1[i] * np.mean(w_aux[i])
        hp = 0.0
        for p in range(molecules.get_n_polymer_types()):
            pol = molecules.get_polymer(p)
            hp -= pol.get_volume_fraction() / pol.get_alpha() * np.log(total_partitions[p])
        return hp + h + self.h_const

    def compute_func_deriv(self, w_aux, phi, indices):
        S = len(self.monomer_types)
        h = np.zeros([len(indices), w_aux.shape[1]], dtype=np.float64)
        for c, i in enumerate(indices):
            if i != S - 1:
                h[c] += 2 * self.h_coef_mu2[i] * w_aux[i]
                h[c] += self.h_coef_mu1[i]
                for j in range(S):
                    h[c] += self.matrix_a[j, i] * phi[self.monomer_types[j]]
            else:
                for j in range(S):
                    h[c] += phi[self.monomer_types[j]]
                h[c] -= 1.0
            if i in self.aux_fields_imag_idx:
                h[c] = -h[c]
        return h


def _setup(params, module, platform):
    """Factory, box, molecules, analyzer and the field theory of a params dict."""
    monomer_types = sorted(params["segment_lengths"].keys())
    chi_n = {}
    for pair, v in params["chi_n"].items():
        mp = sorted(re.split(",| |_|/", pair))
        chi_n[mp[0] + "," + mp[1]] = v
    for mp in itertools.combinations(monomer_types, 2):
        chi_n.setdefault(",".join(sorted(mp)), 0.0)
    mpt = SymmetricPolymerTheory(monomer_types, chi_n)
    factory = module.PlatformSelector.create_factory(platform, False)
    cb = factory.create_computation_box(params["nx"], params["lx"])
    molecules = factory.create_molecules_information(params["chain_model"], params["ds"], params["segment_lengths"])
    for polymer in params["distinct_polymers"]:
        blocks = []
        for b in polymer["blocks"]:
            if "v" in b:
                blocks.append([b["type"], b["length"], b["v"], b["u"]])
            else:
                blocks.append([b["type"], b["length"], len(blocks), len(blocks) + 1])
        molecules.add_polymer(polymer["volume_fraction"], blocks)
    analyzer = factory.create_propagator_analyzer(molecules, params.get("aggregate_propagator_computation", True))
    S = len(monomer_types)
    dt_scaling = np.ones(S)
    for i in range(S - 1):
        dt_scaling[i] = np.abs(mpt.eigenvalues[i]) / np.max(np.abs(mpt.eigenvalues))
    sigma = calculate_sigma(params["langevin"]["nbar"], params["langevin"]["dt"], int(np.prod(params["nx"])),
                            float(np.prod(params["lx"])))
    return monomer_types, chi_n, mpt, factory, cb, molecules, analyzer, dt_scaling, sigma


class LFTS:
    """One L-FTS chain through the public `langevinfts` API (see module doc)."""

    def __init__(self, params, random_seed=None, module=None, platform="cuda"):
        if module is None:
            from langevinfts_b200 import langevinfts as module
        (self.monomer_types, self.chi_n, self.mpt, factory, self.cb, self.molecules, self.analyzer, self.dt_scaling,
         sigma) = _setup(params, module, platform)
        self.solver = factory.create_pseudospectral_solver(self.cb, self.molecules, self.analyzer)
        self.am = factory.create_anderson_mixing(len(self.mpt.aux_fields_imag_idx) * int(np.prod(params["nx"])),
                                                 params["am"]["max_hist"], params["am"]["start_error"],
                                                 params["am"]["mix_min"], params["am"]["mix_init"])
        self.random_bg = np.random.PCG64(random_seed)
        self.random = np.random.Generator(self.random_bg)
        self.langevin = dict(params["langevin"], sigma=sigma)
        self.saddle = dict(params["saddle"])
        self.M = self.cb.get_n_grid()

    def compute_concentrations(self, w_aux):
        w = self.mpt.to_monomer_fields(w_aux)
        self.solver.compute_propagators({t: w[i] for i, t in enumerate(self.monomer_types)})
        self.solver.compute_concentrations()
        return {t: self.solver.get_total_concentration(t) for t in self.monomer_types}

    def find_saddle_point(self, w_aux):
        """lfts.py:807-868; returns (phi, hamiltonian, iterations, error)."""
        S = len(self.monomer_types)
        I = len(self.mpt.aux_fields_imag_idx)
        error_level = 1e20
        hamiltonian = None
        self.am.reset_count()
        for saddle_iter in range(1, self.saddle["max_iter"] + 1):
            phi = self.compute_concentrations(w_aux)
            h_deriv = self.mpt.compute_func_deriv(w_aux, phi, self.mpt.aux_fields_imag_idx)
            old_error_level = error_level
            error_level = np.max(np.std(h_deriv, axis=1))
            if error_level < self.saddle["tolerance"] or saddle_iter == self.saddle["max_iter"]:
                Q = [self.solver.get_total_partition(p) for p in range(self.molecules.get_n_polymer_types())]
                hamiltonian = self.mpt.compute_hamiltonian(self.molecules, w_aux, Q)
            if error_level < self.saddle["tolerance"]:
                break
            for c, i in enumerate(self.mpt.aux_fields_imag_idx):
                h_deriv[c] *= self.dt_scaling[i]
            w_aux[self.mpt.aux_fields_imag_idx] = np.reshape(
                self.am.calculate_new_fields(w_aux[self.mpt.aux_fields_imag_idx], -h_deriv, old_error_level, error_level),
                [I, self.M])
        w_aux[S - 1] -= np.mean(w_aux[S - 1])
        return phi, hamiltonian, saddle_iter, error_level

    def start(self, initial_fields):
        S = len(self.monomer_types)
        w = np.zeros([S, self.M])
        for i in range(S):
            w[i] = np.reshape(initial_fields[self.monomer_types[i]], self.M)
        self.w_aux = self.mpt.to_aux_fields(w)
        self.phi, self.hamiltonian, it, err = self.find_saddle_point(self.w_aux)
        self.noise_prev = np.zeros([self.mpt.R, self.M])
        return it, err

    def step(self):
        """One Langevin step (lfts.py:689-730); returns (iterations, error, H, failed)."""
        w_copy, phi_copy = self.w_aux.copy(), dict(self.phi)
        w_lambda = self.mpt.compute_func_deriv(self.w_aux, self.phi, self.mpt.aux_fields_real_idx)
        noise = self.random.normal(0.0, self.langevin["sigma"], [self.mpt.R, self.M])
        for c, i in enumerate(self.mpt.aux_fields_real_idx):
            s = self.dt_scaling[i]
            self.w_aux[i] += -w_lambda[c] * self.langevin["dt"] * s + 0.5 * (self.noise_prev[c] + noise[c]) * np.sqrt(s)
        self.noise_prev = noise
        phi, h, it, err = self.find_saddle_point(self.w_aux)
        failed = bool(np.isnan(err) or err >= self.saddle["tolerance"])
        if failed:
            self.w_aux, self.phi = w_copy, phi_copy
        else:
            self.phi, self.hamiltonian = phi, h
        return it, err, h, failed


class BatchedLFTS:
    """Many L-FTS replicas on the device-resident batched engine.

    noise="host" (default) draws each step's noise with numpy's
    Generator(PCG64(seed)).normal on the host, exactly as lfts.py:700 does, so
    replica r follows the reference trajectory of its seed.  noise="device"
    draws it on the GPU (lfts_pcg64_normal) from the same PCG64 streams: the
    same raw 64-bit stream, a different normal transform (Box-Muller, not
    numpy's ziggurat), so the noise is N(0, sigma^2) but not the reference's
    sequence.  Checkpoints keep the PCG64 state either way."""

    def __init__(self, params, random_seeds, module=None, platform="cuda", noise="host"):
        if module is None:
            from langevinfts_b200 import langevinfts as module
        (self.monomer_types, self.chi_n, self.mpt, factory, self.cb, self.molecules, self.analyzer, self.dt_scaling,
         self.sigma) = _setup(params, module, platform)
        self.R = len(random_seeds)
        self.M = self.cb.get_n_grid()
        self.S = len(self.monomer_types)
        self.rngs = [np.random.Generator(np.random.PCG64(s)) for s in random_seeds]
        cfg = {
            "monomer_types": self.monomer_types, "matrix_a": list(self.mpt.matrix_a.reshape(-1)),
            "h_coef_mu1": list(self.mpt.h_coef_mu1), "h_coef_mu2": list(self.mpt.h_coef_mu2),
            "h_const": float(self.mpt.h_const), "real_idx": self.mpt.aux_fields_real_idx,
            "imag_idx": self.mpt.aux_fields_imag_idx, "dt_scaling": list(self.dt_scaling),
            "dt": float(params["langevin"]["dt"]), "tolerance": float(params["saddle"]["tolerance"]),
            "max_iter": int(params["saddle"]["max_iter"]), "am_max_hist": int(params["am"]["max_hist"]),
            "am_start_error": float(params["am"]["start_error"]), "am_mix_min": float(params["am"]["mix_min"]),
            "am_mix_init": float(params["am"]["mix_init"]),
        }
        self.engine = module.BatchedLangevin(factory, self.cb, self.molecules, self.analyzer, self.R, cfg)
        self._pool = None
        self.params = params
        self.langevin_step = 0
        if noise not in ("host", "device"):
            raise ValueError('noise must be "host" or "device"')
        self.noise = noise
        if noise == "device":
            self._upload_streams()

    def _upload_streams(self):
        """PCG64 states of the replicas' generators -> the device streams."""
        st = np.zeros([self.R, 4], dtype=np.uint64)
        m64 = (1 << 64) - 1
        for r, g in enumerate(self.rngs):
            s = g.bit_generator.state["state"]
            st[r] = [s["state"] >> 64, s["state"] & m64, s["inc"] >> 64, s["inc"] & m64]
        self.engine.set_noise_streams(st)

    def _download_streams(self):
        """Device stream states -> the replicas' numpy generators (for checkpoints)."""
        st = self.engine.get_noise_streams()
        for r, g in enumerate(self.rngs):
            g.bit_generator.state = {
                "bit_generator": "PCG64",
                "state": {"state": (int(st[r, 0]) << 64) | int(st[r, 1]), "inc": (int(st[r, 2]) << 64) | int(st[r, 3])},
                "has_uint32": 0, "uinteger": 0}

    def start(self, initial_fields):
        """initial_fields: list (per replica) of {monomer type: field}."""
        w_aux = np.zeros([self.R, self.S, self.M])
        for r, f in enumerate(initial_fields):
            w = np.array([np.reshape(f[t], self.M) for t in self.monomer_types])
            w_aux[r] = self.mpt.to_aux_fields(w)
        self.engine.set_fields(w_aux)
        return self.engine.find_saddle_point()

    def draw_noise(self):
        """This step's noise of every replica, drawn from the replica's own PCG64
        stream exactly as lfts.py:700 draws it (threads overlap the draws)."""
        nR = self.mpt.R
        out = np.empty([self.R, nR, self.M])
        if self._pool is None:
            from concurrent.futures import ThreadPoolExecutor
            self._pool = ThreadPoolExecutor(max_workers=8)

        def one(r):
            out[r] = self.rngs[r].normal(0.0, self.sigma, [nR, self.M])
        list(self._pool.map(one, range(self.R)))
        return out

    def step(self, noise=None, start=None):
        """One Langevin step of every replica.  start (optional): a callable
        (e.g. learned.LearnedStart) run after the Langevin update and before the
        saddle-point search; it may change the imaginary fields on the device,
        which the search then starts from.  A start with a before_update method
        gets it called before the update."""
        if start is not None:
            import torch
            keep = None
            if hasattr(start, "before_update"):
                start.before_update(self)
            if self.noise == "device" and noise is None:
                self.engine.langevin_update_rng(self.sigma)
            else:
                if noise is None:
                    noise = self.draw_noise()
                with torch.cuda.stream(torch.cuda.ExternalStream(self.engine.stream_ptr())):
                    keep = torch.from_numpy(np.ascontiguousarray(noise)).cuda()
                self.engine.langevin_update_device(keep.data_ptr())
            start(self)
            stats = self.engine.finish_step()
            del keep
            self.langevin_step += 1
            return stats
        if noise is None and self.noise == "device":
            stats = self.engine.step_rng(self.sigma)
            self.langevin_step += 1
            return stats
        if noise is None:
            noise = self.draw_noise()
        stats = self.engine.step(noise)
        self.langevin_step += 1
        return stats

    def step_device(self, noise_ptr, start=None):
        """One Langevin step with this step's noise already on the device (a
        pointer to [R][n_real][M] doubles); start as in step()."""
        if start is None:
            stats = self.engine.step_device(noise_ptr)
        else:
            if hasattr(start, "before_update"):
                start.before_update(self)
            self.engine.langevin_update_device(noise_ptr)
            start(self)
            stats = self.engine.finish_step()
        self.langevin_step += 1
        return stats

    def fields(self):
        return self.engine.get_fields(self.S)

    def save_simulation_data(self, paths):
        """Write one checkpoint per replica, paths[r], with the keys and layout of
        the reference driver's save_simulation_data (lfts.py:569-600): monomer
        fields, concentrations, the replica's PCG64 state, the step count and
        the previous step's noise.  Either driver can continue from it."""
        from scipy.io import savemat
        if len(paths) != self.R:
            raise ValueError("one path per replica")
        if self.noise == "device":
            self._download_streams()
        w_aux = self.fields()
        phi = self.engine.get_concentrations(self.S)
        noise_prev = self.engine.get_noise_prev()
        for r, path in enumerate(paths):
            w = self.mpt.to_monomer_fields(w_aux[r])
            state = self.rngs[r].bit_generator.state
            mdic = {
                "initial_params": self.params,
                "dim": self.cb.get_dim(), "nx": self.cb.get_nx(), "lx": self.cb.get_lx(),
                "monomer_types": self.monomer_types, "chi_n": dict(self.chi_n),
                "chain_model": self.params["chain_model"], "ds": self.params["ds"],
                "dt": self.params["langevin"]["dt"], "nbar": self.params["langevin"]["nbar"],
                "eigenvalues": self.mpt.eigenvalues,
                "aux_fields_real": self.mpt.aux_fields_real_idx, "aux_fields_imag": self.mpt.aux_fields_imag_idx,
                "matrix_a": self.mpt.matrix_a, "matrix_a_inverse": self.mpt.matrix_a_inv,
                "langevin_step": self.langevin_step,
                "random_generator": state["bit_generator"],
                "random_state_state": str(state["state"]["state"]),
                "random_state_inc": str(state["state"]["inc"]),
                "normal_noise_prev": noise_prev[r]}
            for i, name in enumerate(self.monomer_types):
                mdic["w_" + name] = w[i]
                mdic["phi_" + name] = phi[r, i]
            savemat(path, mdic, long_field_names=True, do_compression=True)

    def continue_run(self, paths):
        """Resume every replica from a checkpoint (lfts.py:602-629): restore its
        PCG64 state, fields and previous noise, then find the saddle point as
        the reference's run() does before its first step.  Returns those
        statistics; the next step() is step langevin_step + 1."""
        from scipy.io import loadmat
        if len(paths) != self.R:
            raise ValueError("one path per replica")
        fields, noise_prev, steps = [], np.zeros([self.R, self.mpt.R, self.M]), set()
        for r, path in enumerate(paths):
            d = loadmat(path, squeeze_me=True)
            self.rngs[r].bit_generator.state = {
                "bit_generator": "PCG64",
                "state": {"state": int(d["random_state_state"]), "inc": int(d["random_state_inc"])},
                "has_uint32": 0, "uinteger": 0}
            fields.append({name: np.array(d["w_" + name]) for name in self.monomer_types})
            noise_prev[r] = np.reshape(d["normal_noise_prev"], [self.mpt.R, self.M])
            steps.add(int(d["langevin_step"]))
        if len(steps) != 1:
            raise ValueError("the checkpoints are at different Langevin steps")
        stats = self.start(fields)
        self.engine.set_noise_prev(noise_prev)
        if self.noise == "device":
            self._upload_streams()
        self.langevin_step = steps.pop()
        return stats

    def sf_pairs(self):
        """Monomer-type index pairs of the structure function, in the order
        lfts.py:665-668 builds its dictionary."""
        import itertools
        return [tuple(sorted(p)) for p in itertools.combinations_with_replacement(range(self.S), 2)]

    def accumulate_structure_function(self):
        """Add this step's <u(k) phi(-k)> of every replica to the device sums
        (lfts.py:753-767): phi_i and the auxiliary fields 0..S-2 are transformed
        on the device, mu_i = sum_k F[w_aux_k] A_inv[k, i] / eigenvalue_k / M."""
        coef = np.array([[self.mpt.matrix_a_inv[k, i] / self.mpt.eigenvalues[k] / self.M for i in range(self.S)]
                         for k in range(self.S - 1)], dtype=np.float64).reshape(max(self.S - 1, 1), self.S)
        self.engine.sf_accumulate(np.ascontiguousarray(coef), [v for p in self.sf_pairs() for v in p])

    def structure_function(self, reset=True):
        """The accumulated sums, {"A,B": complex [R, nx, ny, nz//2+1]} (the
        reference's sf_average before its recording scale, lfts.py:780-782)."""
        nx = list(self.cb.get_nx())
        shape_k = nx[:-1] + [nx[-1] // 2 + 1]
        sf = self.engine.get_structure_function(shape_k, reset)
        return {self.monomer_types[a] + "," + self.monomer_types[b]: sf[:, p] for p, (a, b) in enumerate(self.sf_pairs())}

    def h_deriv_chin(self, stats):
        """dH/dchiN of every replica (lfts.py:265-274) from the field moments that
        find_saddle_point / step return."""
        mean = np.reshape(stats["aux_mean"], [self.R, self.S])
        msq = np.reshape(stats["aux_msq"], [self.R, self.S])
        out = []
        for r in range(self.R):
            dH = {}
            for key in self.chi_n:
                dH[key] = self.mpt.h_const_deriv_chin[key]
                for i in range(self.S - 1):
                    dH[key] += self.mpt.h_coef_mu2_deriv_chin[key][i] * msq[r, i]
                    dH[key] += self.mpt.h_coef_mu1_deriv_chin[key][i] * mean[r, i]
            out.append(dH)
        return out
