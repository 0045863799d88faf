"""numpy restatement of molecular2's RHF driver — TEST INFRASTRUCTURE ONLY.

Follows, step for step:
  * SCF::rhf                     src/scf.cpp:90-185 (loop, convergence test)
  * SCF::calcE / calcErr         src/scf.cpp:29-58
  * DIISEngine::compute / solve  src/diis.cpp:22-116 (incl. the rank fallback;
    the damping scale is overwritten by the j=i store there, so it has no
    effect and is not applied here either)
  * Fock::makeFock(P, mult)      src/fockbuild.cpp:176-222 (incremental Fock,
    resets), Fock::average / transform / diagonalise / makeDens
                                 src/fock.cpp:144-244
  * Fock::compute_soad_guess     src/fock.cpp:174-225
  * Fock::compute_forces         src/rhfgrad.cpp:15-89
The two-electron builds are injected (``jk`` callables) so the same driver can
run on the oracle's CPU J/K or, in tests, compare against the GPU engine.
"""
import numpy as np

from . import F, jk_direct, schwarz, one_body, fock_general, df_jk, one_body_deriv, grad2e


class DIIS:
    def __init__(self, maxdiis=8, use=True):
        self.max = maxdiis if maxdiis > 0 else 8
        self.use = use
        self.errs = []
        self.lastB = np.zeros((1, 1))

    def compute(self, errors):
        weights = np.zeros(0)
        it = len(self.errs) + 1
        if not self.use:
            return weights
        if it > self.max:
            self.errs.pop(0)
        new = np.concatenate(errors)
        self.errs.append(new)
        if it == 1:
            self.lastB[0, 0] = new @ new
        if it > 1:
            lim = min(it, self.max)
            B = np.zeros((lim + 1, lim + 1))
            start = 1 if it > lim else 0
            for i in range(lim - 1):
                for j in range(i, lim - 1):
                    B[i, j] = self.lastB[i + start, j + start]
                    B[j, i] = B[i, j]
                B[lim, i] = B[i, lim] = -1.0
            for i in range(lim):
                B[lim - 1, i] = self.errs[i] @ self.errs[lim - 1]
                B[i, lim - 1] = B[lim - 1, i]
            B[lim, lim - 1] = B[lim - 1, lim] = -1.0
            self.lastB = B
            weights = self._solve(B, 0)
            rank = int(weights[-1])
            start = 1
            while rank < (lim - start + 1) and start < lim:
                weights = self._solve(B, start)
                start += 1
                rank = int(weights[-1])
            weights = weights[:-2]
        return weights

    @staticmethod
    def _solve(B, start):
        size = B.shape[0] - start
        norm = 1.0
        if B[start, start] > 1e-10:
            norm = 1.0 / B[start, start]
        nB = np.zeros((size, size))
        for i in range(size - 1):
            for j in range(i, size - 1):
                nB[i, j] = nB[j, i] = norm * B[i + start, j + start]
            nB[i, size - 1] = nB[size - 1, i] = -1.0
        w = np.zeros(size)
        w[-1] = -1.0
        sv = np.linalg.svd(nB, compute_uv=False)
        rank = int(np.sum(sv > sv[0] * np.finfo(float).eps * size)) if sv.size else 0
        try:
            x = np.linalg.solve(nB, w)
        except np.linalg.LinAlgError:
            x = np.linalg.lstsq(nB, w, rcond=None)[0]
        return np.concatenate([x, [rank]])


class RHF:
    """One RHF calculation: state of ``Fock`` + ``SCF`` for the closed-shell case."""

    def __init__(self, basis, jk=None, df=None, guess="soad", maxdiis=8, diis=True, precision=1e-12,
                 maxiter=40, enconverge=1e-7, densconverge=1e-4, minbasis=None, nthreads=None):
        self.basis = basis
        mol = basis.mol
        self.mol = mol
        self.n = basis.nbf
        self.nocc = mol.nocc
        self.S, T, V = one_body(basis)
        self.hcore = T + V
        lam, U = np.linalg.eigh(self.S)
        self.orthog = U @ np.diag(1.0 / np.sqrt(lam)) @ U.T
        self.precision = precision
        self.Q = schwarz(basis)
        self.df = df  # None or a callable Cocc -> (J, K) w.r.t. C C^T
        self.jk = jk or (lambda D: jk_direct(basis, D, self.Q, self.precision, 1.0, nthreads)[:2])
        self.guess = guess
        self.minbasis = minbasis
        self.maxiter = maxiter
        self.E_CONV = enconverge
        self.D_CONV = densconverge
        self.diis_on = diis
        self.diis = DIIS(maxdiis, diis)
        self.MAX = maxdiis
        self.focks = []
        self.iter = 0
        self.rms_error = 1.0
        self.started_incremental = False
        self.reset_incremental = False
        self.next_reset = 0.0
        self.last_reset = 0
        self.incremental_threshold = 1e-5
        self.dens = None
        self.dens_diff = None
        self.energy = 0.0
        self.last_energy = 0.0
        self.jk_builds = 0
        self.history = []

    # --- Fock -------------------------------------------------------------
    def soad_fock(self):
        G = fock_general(self.basis, self.minbasis, self.minbasis_density, shelldiag=True)
        return self.hcore + G

    def transform(self, first):
        if first:
            if self.guess == "hcore":
                self.fockm = self.orthog.T @ self.hcore @ self.orthog
                self.fockinc = self.hcore.copy()
                self.focka = self.hcore.copy()
            else:
                self.focka = self.soad_fock()
                self.fockinc = self.focka.copy()
                self.fockm = self.orthog.T @ self.focka @ self.orthog
        else:
            self.fockm = self.orthog.T @ self.focka @ self.orthog

    def diagonalise(self):
        eps, U = np.linalg.eigh(self.fockm)
        self.CP = self.orthog @ U
        self.eps = eps

    def make_dens(self):
        if self.dens is not None:
            self.dens_diff = -self.dens
        C = self.CP[:, :self.nocc]
        self.dens = 2.0 * C @ C.T
        if self.dens_diff is None:
            self.dens_diff = self.dens.copy()
        else:
            self.dens_diff = self.dens_diff + self.dens

    def make_jk(self, P):
        self.jk_builds += 1
        if self.df is not None:
            J, K = self.df(P)
            return 2.0 * J - K
        J, K = self.jk(P)
        return J - 0.5 * K

    def make_fock(self):
        if self.df is None:
            self.focka = self.fockinc
            if (not self.started_incremental) and self.rms_error < self.incremental_threshold:
                self.started_incremental = True
                self.reset_incremental = False
                self.next_reset = self.rms_error / 1e1
                self.last_reset = self.iter - 1
            if self.reset_incremental or not self.started_incremental:
                self.focka = self.hcore
                self.dens_diff = self.dens.copy()
            if self.reset_incremental and self.started_incremental:
                self.reset_incremental = False
                self.last_reset = self.iter
                self.next_reset = self.rms_error / 1e1
            self.focka = self.focka + self.make_jk(self.dens_diff)
            self.fockinc = self.focka
        else:
            self.focka = self.hcore + self.make_jk(self.CP[:, :self.nocc])
        if self.diis_on:
            if self.iter >= self.MAX:
                self.focks.pop(0)
            self.focks.append(self.focka)
            self.iter += 1

    def average(self, w):
        if self.diis_on and self.iter > 2:
            off = len(self.focks) - len(w)
            self.focka = sum(w[i - off] * self.focks[i] for i in range(off, len(self.focks)))

    # --- SCF --------------------------------------------------------------
    def calc_err(self):
        F_, D, S = self.focka, self.dens, self.S
        e = F_ @ (D @ S) - S @ (D @ F_)
        e = self.orthog.T @ e @ self.orthog
        self.error = np.linalg.norm(e)
        return e.reshape(-1, order="F")

    def calc_e(self):
        self.last_energy = self.energy
        one = 0.5 * np.trace(self.dens @ self.hcore)
        two = 0.5 * np.trace(self.dens @ self.focka) - one
        self.energy = 2.0 * one + two + self.mol.enuc()

    def run(self):
        if self.guess != "hcore" and self.minbasis_density is None:
            raise ValueError("SOAD guess needs the minimal basis")
        self.transform(True)
        self.diagonalise()
        self.make_dens()
        old = self.dens.copy()
        self.make_fock()
        weights = self.diis.compute([self.calc_err()])
        self.calc_e()
        self.history.append((0, self.energy, 0.0, 0.0))
        self.average(weights)
        self.transform(False)
        it = 1
        converged = False
        while not converged and it < self.maxiter:
            self.diagonalise()
            self.make_dens()
            dd = np.linalg.norm(self.dens - old)
            old = self.dens.copy()
            self.make_fock()
            err = self.calc_err()
            self.rms_error = np.linalg.norm(err) / (self.n * self.n)
            if self.rms_error < self.next_reset or it - self.last_reset > 8:
                self.reset_incremental = True
            if it > 2:
                weights = self.diis.compute([err])
            self.calc_e()
            delta = abs(self.energy - self.last_energy)
            self.history.append((it, self.energy, delta, dd))
            if it > 2:
                self.average(weights)
            self.transform(False)
            converged = dd < self.D_CONV and delta < self.E_CONV
            it += 1
        self.diagonalise()
        self.converged = converged
        self.iterations = it
        return self.energy

    @property
    def minbasis_density(self):
        if self.minbasis is None:
            return None
        from molecular2_b200.basis import sto3g_density
        return sto3g_density(self.mol)

    # --- gradient (Fock::compute_forces) ------------------------------------
    def forces(self):
        mol = self.mol
        na = mol.natom
        D = self.dens
        T1, V1, S1 = None, None, None
        S1, T1, V1 = one_body_deriv(self.basis)
        C = self.CP[:, :self.nocc]
        W = C @ np.diag(self.eps[:self.nocc]) @ C.T
        F1 = np.array([np.sum((T1[i] + V1[i]) * D) for i in range(3 * na)]).reshape(na, 3)
        Fp = -np.array([2.0 * np.sum(S1[i] * W) for i in range(3 * na)]).reshape(na, 3)
        F2 = grad2e(self.basis, D, self.Q, self.precision)
        return F1 + Fp + F2 + mol.enuc_grad()
