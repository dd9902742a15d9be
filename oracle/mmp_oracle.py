"""FP64 numpy restatement of alexandreroget/MM_Propagation's CPU solver.

TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT. Only tests/, the smoke check in
__graft_entry__.py and bench.py's CPU-baseline leg may import this module, and
only as the checker. The product (mm_propagation_b200, libmmp_b200.so) never
imports it and has no CPU fallback.

Each function restates one piece of the reference, which is cited by
path:line within that project. The restatement follows the reference's data
flow exactly (time-domain state, cumulative-product Lawson exponentials,
slot-indexed pair products), including the behaviours this project calls
"quirks" and reproduces on the device for parity:

* the k=2 and k>=3 dispersion signs (src/MultimodePropagation.cpp:165-187);
* z reset to 0 at every computeLawsonRK call (src/MultimodePropagation.cpp:158-163);
* V[slot] built from U[slot % M] * conj(U[slot / M]) rather than from
  unique_pairs[slot] (src/MultimodePropagation_CPU.cpp:126-133, :195-205);
* nz = floor(z_final / delta_z) in the no-argument computeLawsonRK
  (src/MultimodePropagation.cpp:213-216).

Pinning: the reference has no tests or golden vectors. This restatement is
pinned against the reference's own code compiled here (oracle/_ref/libmmref.so,
built by oracle/Makefile from the unmodified sources) through fixtures in
tests/golden/ generated by tests/golden/make_golden.py.
"""
from __future__ import annotations

import math

import numpy as np

# ---- Butcher tableaus: src/RungeKutta.cpp ------------------------------------------------

S21 = math.sqrt(21.0)


def butcher4():
    """Classic RK4 (src/RungeKutta.cpp:3-21)."""
    a = [[0.0], [0.5], [0.0, 0.5], [0.0, 0.0, 1.0]]
    b = [1 / 6.0, 1 / 3.0, 1 / 3.0, 1 / 6.0]
    c = [0.0, 0.5, 0.5, 1.0]
    return a, b, c


def butcher7(nu: float = 1.0):
    """7-stage order-6 family in nu (src/RungeKutta.cpp:24-72); the solver uses nu = 1."""
    a = [
        [0.0],
        [nu],
        [(4 * nu - 1) / (8 * nu), 1 / (8 * nu)],
        [(10 * nu - 2) / (27 * nu), 2 / (27 * nu), (8 * nu) / (27 * nu)],
        [(56 - 77 * nu + (8 - 17 * nu) * S21) / (392 * nu), (-8 * (7 + S21)) / (392 * nu),
         (48 * (7 + S21) * nu) / (392 * nu), (-3 * (21 + S21) * nu) / (392 * nu)],
        [(-5 * (287 * nu - 56 - (59 * nu - 8) * S21)) / (1960 * nu), (-40 * (7 - S21)) / (1960 * nu),
         (320 * S21 * nu) / (1960 * nu), (3 * (21 - 121 * S21) * nu) / (1960 * nu),
         (392 * (6 - S21) * nu) / (1960 * nu)],
        [(15 * ((30 * nu - 8) - 7 * nu * S21)) / (180 * nu), 120 / (180 * nu),
         (-40 * (5 + 7 * S21) * nu) / (180 * nu), (63 * (2 + 3 * S21) * nu) / (180 * nu),
         (-14 * (49 - 9 * S21) * nu) / (180 * nu), (70 * (7 + S21) * nu) / (180 * nu)],
    ]
    b = [9 / 180, 0.0, 64 / 180, 0.0, 49 / 180, 49 / 180, 9 / 180]
    c = [0.0, nu, 0.5, 2 / 3.0, (7 + S21) / 14, (7 - S21) / 14, 1.0]
    return a, b, c


def butcher7_lambda_mu(lam: float, mu: float):
    """7-stage family in (lambda, mu) (src/RungeKutta.cpp:75-122); never selected by
    the reference's solver, reachable here through rk_variant."""
    a = [
        [0.0],
        [mu],
        [2 / 3 - 2 / (9 * mu), 2 / (9 * mu)],
        [5 / 12 - 1 / (9 * mu), 1 / (9 * mu), -1 / 12],
        [17 / 16 - 3 / (8 * mu), 3 / (8 * mu), -3 / 16, -3 / 8],
        [17 / 16 - 3 / (8 * mu) + 1 / (4 * lam), 3 / (8 * mu), -3 / 16 - 3 / (4 * lam),
         -3 / 8 - 3 / (2 * lam), 2 / lam],
        [-27 / 44 + 3 / (11 * mu), -3 / (11 * mu), 63 / 44, 18 / 11, 4 * ((lam - 4) / 11),
         -(4 * lam) / 11],
    ]
    b = [1 / 120, 0.0, 27 / 40, 27 / 40, (lam - 8) / 15, -lam / 15, 11 / 120]
    c = [0.0, mu, 2 / 3, 1 / 3, 0.5, 0.5, 1.0]
    return a, b, c


def butcher11():
    """11-stage order-8 tableau (src/RungeKutta.cpp:125-175)."""
    s = S21
    a = [
        [0.0],
        [0.5],
        [0.25, 0.25],
        [1 / 7, (-7 + 3 * s) / 98, (21 - 5 * s) / 49],
        [(11 - s) / 84, 0.0, (18 - 4 * s) / 63, (21 + s) / 252],
        [(5 - s) / 48, 0.0, (9 - s) / 36, (-231 - 14 * s) / 360, (63 + 7 * s) / 80],
        [(10 + s) / 42, 0.0, (-432 - 92 * s) / 315, (633 + 145 * s) / 90, (-504 - 115 * s) / 70,
         (63 + 13 * s) / 35],
        [1 / 14, 0.0, 0.0, 0.0, (14 + 3 * s) / 126, (13 + 3 * s) / 63, 1 / 9],
        [1 / 32, 0.0, 0.0, 0.0, (91 + 21 * s) / 576, 11 / 72, (-385 + 75 * s) / 1152,
         (63 - 13 * s) / 128],
        [1 / 14, 0.0, 0.0, 0.0, 1 / 9, (-733 + 147 * s) / 2205, (515 - 111 * s) / 504,
         (-51 + 11 * s) / 56, (132 - 28 * s) / 245],
        [0.0, 0.0, 0.0, 0.0, (-42 - 7 * s) / 18, (-18 - 28 * s) / 45, (-273 + 53 * s) / 72,
         (301 - 53 * s) / 72, (28 + 28 * s) / 45, (49 + 7 * s) / 18],
    ]
    b = [1 / 20, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 49 / 180, 16 / 45, 49 / 180, 1 / 20]
    c = [0.0, 0.5, 0.5, (7 - s) / 14, (7 - s) / 14, 0.5, (7 + s) / 14, (7 + s) / 14, 0.5,
         (7 - s) / 14, 1.0, 1.0]
    return a, b, c


def select_tableau(method_order: int, rk_variant: int = 0, lam: float = 0.0, mu: float = 0.0):
    """setRungeKuttaCoefficients (src/MultimodePropagation.cpp:15-27): 8 -> Butcher11,
    6 -> Butcher7(nu=1), anything else -> RK4."""
    if rk_variant == 1:
        return butcher7_lambda_mu(lam, mu)
    if method_order == 8:
        return butcher11()
    if method_order == 6:
        return butcher7(1.0)
    return butcher4()


# ---- FFT conventions: src/DiscreteFourierTransform.cpp --------------------------------------

def fft(x):
    """Forward_DFT: FFTW_FORWARD, unnormalised (src/DiscreteFourierTransform.cpp:24-26)."""
    return np.fft.fft(x, axis=-1)


def ifft(x):
    """Inverse_DFT: FFTW_BACKWARD then * 1/n (src/DiscreteFourierTransform.cpp:32-38)."""
    return np.fft.ifft(x, axis=-1)


# ---- the solver --------------------------------------------------------------------------

class OracleSolver:
    """MultimodePropagationCPU_RamanOFF / _RamanON restated.

    `prob` is an mm_propagation_b200.workloads.Problem (plain numpy data).
    `physical_pairs` switches the pair table to unique_pairs[slot] (what the
    reference's GPU backend does, src/MultimodePropagation_GPU.cu:189-193); the
    default reproduces the CPU backend.
    """

    def __init__(self, prob, physical_pairs: bool = False):
        self.M = M = prob.n_modes
        self.nt = nt = prob.nt
        self.raman = bool(prob.raman)
        # MultimodePropagation(in): src/MultimodePropagation.cpp:4-12
        self.a, self.b, self.c = select_tableau(prob.method_order, prob.rk_variant,
                                                prob.rk_lambda, prob.rk_mu)
        self.s = len(self.b)
        self.T0 = prob.pulse_width
        # setDimensionlessVariables: src/MultimodePropagation.cpp:31-56
        gamma = prob.nonlinearity_const
        self.sign_gamma = 1.0 if gamma >= 0 else -1.0
        beta = np.asarray(prob.dispersion, dtype=np.float64)
        max_beta2 = float(np.max(np.abs(beta[:, 2])))                        # :67-77
        Q = prob.coupling
        max_Q = float(np.max(np.abs(Q["value"]))) if len(Q) else 0.0         # :81-97
        LD = self.T0 * self.T0 / max_beta2                                   # :42
        n_beta = beta.shape[1]
        cfac = np.array([1.0 / self.T0 ** i * LD for i in range(n_beta)])   # :100-114
        self.beta_tilde = beta * cfac[None, :]
        self.Q_tilde = [[(int(e["k"]), int(e["l"]), int(e["m"]), float(e["value"]) / max_Q)
                         for e in Q[Q["p"] == p]] for p in range(M)]         # :117-136
        self.t_final = prob.time_window / self.T0                            # :47
        self.delta_t = self.t_final / nt
        self.z_final = prob.fiber_length / LD                                # :50
        self.delta_z = self.z_final / prob.n_steps
        self.conversion_factor = math.sqrt(abs(gamma) * LD) * math.sqrt(max_Q)  # :53
        self.LD, self.max_Q, self.max_beta2 = LD, max_Q, max_beta2
        self.psi = np.asarray(prob.initial_fields, dtype=np.complex128) * self.conversion_factor
        # setUniquePairs: src/MultimodePropagation.cpp:139-155 (p outer, insertion order inner)
        self.unique_pairs = []
        for p in range(M):
            for (k, l, m, v) in self.Q_tilde[p]:
                code = l + m * M
                if code not in self.unique_pairs:
                    self.unique_pairs.append(code)
        self.physical_pairs = physical_pairs
        if self.raman:
            # MultimodePropagationCPU_RamanON: src/MultimodePropagation_CPU.cpp:170-176
            self.fR = prob.raman_proportion
            self.hR_fft = fft(np.asarray(prob.raman_response, dtype=np.float64).astype(np.complex128))
        self.z = 0.0

    # initLawsonRK + computeLinearOperators + initExponentialOperatorsMatrix
    def _init_lawson(self):
        """src/MultimodePropagation.cpp:158-199."""
        self.z = 0.0
        nt = self.nt
        j = np.arange(nt)
        k = np.where(j <= nt // 2, j, j - nt)
        alpha = (2 * math.pi / self.t_final) * k
        bt = self.beta_tilde
        n_beta = bt.shape[1]
        L = 1j * (bt[:, 0:1] - bt[:, 1:2] * alpha[None, :] - bt[:, 2:3] / 2 * (alpha * alpha)[None, :])
        for kk in range(3, n_beta):
            L = L + 1j * (((-1.0) ** kk) * bt[:, kk:kk + 1] / math.factorial(kk) * alpha[None, :] ** kk)
        self.L = L
        self.E1 = np.exp(L * self.delta_z)
        self.E = [np.exp(L * (ci * self.delta_z)) for ci in self.c]

    def pair_fields(self, U):
        """Step 2 of computeNonlinearity: V[slot] (src/MultimodePropagation_CPU.cpp:126-133)."""
        M = self.M
        V = []
        for slot, code in enumerate(self.unique_pairs):
            src = code if self.physical_pairs else slot
            l, m = src % M, src // M
            V.append(U[l] * np.conj(U[m]))
        return V

    def nonlinearity(self, E_i, psi_i):
        """computeNonlinearity, Raman OFF (src/MultimodePropagation_CPU.cpp:111-166)
        and Raman ON (:180-238)."""
        U = ifft(fft(psi_i) * E_i)                                     # step 1
        V = self.pair_fields(U)                                        # step 2
        if self.raman:
            VR = [ifft(fft(v) * self.hR_fft) * self.delta_t for v in V]   # :241-251
        slot_of = {code: i for i, code in enumerate(self.unique_pairs)}
        sigma = np.zeros_like(psi_i)
        for p in range(self.M):                                        # step 3
            acc = np.zeros(self.nt, dtype=np.complex128)
            for (k, l, m, q) in self.Q_tilde[p]:
                lm = slot_of[l + m * self.M]
                if self.raman:
                    W = V[lm] * (q * (1 - self.fR)) + VR[lm] * (q * self.fR * self.T0)
                else:
                    W = V[lm] * q
                acc += W * U[k]
            sigma[p] = acc
        N = ifft(fft(sigma) * np.conj(E_i)) * (1j * self.sign_gamma)   # step 4
        return N

    def apply_rk(self, h):
        """applyRungeKuttaMethod (src/MultimodePropagation_CPU.cpp:47-85)."""
        N = []
        result = self.psi.copy()
        for i in range(self.s):
            psi_i = self.psi.copy()
            for j in range(i):
                if self.a[i][j] != 0.0:
                    psi_i = psi_i + N[j] * (self.a[i][j] * h)
            Ni = self.nonlinearity(self.E[i], psi_i)
            N.append(Ni)
            if self.b[i] != 0.0:
                result = result + Ni * (self.b[i] * h)
        self.psi = result

    def compute_lawson_rk(self, nz=None):
        """computeLawsonRK(nz) (src/MultimodePropagation_CPU.cpp:24-34); with nz None,
        the no-argument form nz = floor(z_final / delta_z) (src/MultimodePropagation.cpp:213-216)."""
        if nz is None:
            nz = int(math.floor(self.z_final / self.delta_z))
        self._init_lawson()
        for _ in range(nz):
            self.apply_rk(self.delta_z)
            for i in range(self.s):                                     # :37-44
                self.E[i] = self.E[i] * self.E1
            self.z += self.delta_z

    def continue_lawson_rk(self, nz):
        """nz more steps from the current z, without the reset of initLawsonRK: the
        stage exponentials are rebuilt at z (E_i = exp(L (z + c_i h))) and the steps run
        as in computeLawsonRK. What a correct chunked propagation does."""
        if not hasattr(self, "L"):
            self._init_lawson()
        self.E = [np.exp(self.L * (self.z + ci * self.delta_z)) for ci in self.c]
        for _ in range(nz):
            self.apply_rk(self.delta_z)
            for i in range(self.s):
                self.E[i] = self.E[i] * self.E1
            self.z += self.delta_z

    def get_result(self):
        """getResult (src/MultimodePropagation_CPU.cpp:88-104)."""
        if not hasattr(self, "L"):
            self._init_lawson()
        return ifft(fft(self.psi) * np.exp(self.L * self.z)) / self.conversion_factor


def solve(prob, chunks=None, physical_pairs=False):
    """Construct, run computeLawsonRK for each chunk (None entries mean the
    no-argument form), return getResult() as complex128 [M][NT]."""
    sol = OracleSolver(prob, physical_pairs=physical_pairs)
    for nz in (chunks if chunks is not None else [prob.n_steps]):
        sol.compute_lawson_rk(nz)
    return sol.get_result()


def coupling_from_dense(q):
    """setCouplingCoefficients (matlab/mm_propagation.cpp:186-209): walk the dense
    M^4 array in MATLAB element order (p fastest, then k, l, m) and append every
    non-zero (k, l, m, value) to Q^(p). Returns [(p, k, l, m, value)] in that order."""
    q = np.asarray(q, dtype=np.float64)
    M = q.shape[0]
    out = []
    for m in range(M):
        for l in range(M):
            for k in range(M):
                for p in range(M):
                    v = float(q[p, k, l, m])
                    if v != 0.0:
                        out.append((p, k, l, m, v))
    return out


def abs_text_lines(phi0, phi):
    """simulations/main.cpp:101-103: per sample, |phi0_p| then |phi_p| for every mode,
    joined by " ; ", numbers as the default iostream prints them (%g)."""
    cols = [np.abs(a) for a in (list(phi0) if phi0 is not None else []) + list(phi)]
    return [" ; ".join("%g" % c[i] for c in cols) for i in range(len(cols[0]))]


def snapshots(prob, n_save, z_mode=0):
    """The MEX front end's n_save loop (matlab/mm_propagation.cpp:61-91): n_save - 1
    chunks of n_steps // n_save steps, then one of n_steps // n_save + n_steps % n_save,
    getResult after each, Z += nz * fiber_length / n_steps. z_mode 1 calls
    computeLawsonRK per chunk (z restarts at 0 each time, as the reference does);
    z_mode 0 continues z across chunks. Returns (fields [n_save][M][NT], Z [n_save])."""
    sol = OracleSolver(prob)
    nz = prob.n_steps // n_save
    delta_Z = prob.fiber_length / prob.n_steps
    out, Z, z_acc = [], [], 0.0
    for i in range(n_save):
        n = nz if i < n_save - 1 else nz + prob.n_steps % n_save
        if z_mode == 1 or i == 0:
            sol.compute_lawson_rk(n)
        else:
            sol.continue_lawson_rk(n)
        out.append(sol.get_result())
        z_acc += n * delta_Z
        Z.append(z_acc)
    return np.stack(out), np.array(Z)


def rel_l2_per_mode(x, ref):
    """||x_p - ref_p||_2 / ||ref_p||_2 for each mode p."""
    x = np.asarray(x)
    ref = np.asarray(ref)
    num = np.sqrt((np.abs(x - ref) ** 2).sum(axis=-1))
    den = np.sqrt((np.abs(ref) ** 2).sum(axis=-1))
    return num / np.where(den > 0, den, 1.0)
