"""Impurity models of the benchmark workloads, built on the host with ``atom_diag``.

Every builder returns a :class:`Model` holding the Fock-space blocks, the symmetry-set field
operators, the atomic pseudo-particle propagator on the DLR nodes and the hybridization as DLR
poles and coefficients.  The DLR nodes come from the caller (``rf`` dimensionless real
frequencies, ``it`` relative-format imaginary-time nodes), so one model can be evaluated on any
basis.  Orbital index ``i`` of an ``M``-orbital spinful model is spin ``i // M`` (0 = up) and
orbital ``i % M``, the flattening of ``gf_struct = [('up', M), ('dn', M)]`` used by
``BlockSparseSolver.__from_blockgf_to_dense`` (``python/triqs_xca/block_sparse_solver.py:188-204``).
"""

import itertools
from dataclasses import dataclass, field

import numpy as np

from .atom_diag import AtomDiag, FockSpace, atomic_pseudo_particle_greens_function, get_operators


def kernel(t, om):
    """cppdlr's signed fermionic kernel K(t, om) = -exp(-t om)/(1 + exp(-om)) in relative time format."""
    t = np.asarray(t, dtype=float)
    om = np.asarray(om, dtype=float)
    t, om = np.broadcast_arrays(t, om)
    neg = t < 0
    tt = np.where(neg, -t, t)
    oo = np.where(neg, -om, om)
    pos = oo >= 0
    a = np.exp(-tt * np.where(pos, oo, 0.0)) / (1.0 + np.exp(-np.where(pos, oo, 0.0)))
    b = np.exp((1.0 - tt) * np.where(pos, 0.0, oo)) / (1.0 + np.exp(np.where(pos, 0.0, oo)))
    return -np.where(pos, a, b)


def rel2abs(t):
    t = np.asarray(t, dtype=float)
    return np.where(t < 0, 1.0 + t, t)


@dataclass
class Model:
    name: str
    beta: float
    lam: float
    eps: float
    n: int
    ad: AtomDiag
    dims: np.ndarray
    labels: np.ndarray
    F_index: np.ndarray
    F_blocks: list
    Fd_index: np.ndarray
    Fd_blocks: list
    rf: np.ndarray
    it: np.ndarray
    G0: list
    eta0: float
    hyb_poles: np.ndarray          # physical units (the evaluator multiplies by beta)
    hyb_coeffs: np.ndarray         # (p, n, n) complex
    extra: dict = field(default_factory=dict)

    @property
    def r(self):
        return len(self.it)

    @property
    def tau(self):
        return self.beta * rel2abs(self.it)


def vals2coefs(rf, it, vals):
    K = kernel(np.asarray(it)[:, None], np.asarray(rf)[None, :])
    shp = vals.shape
    return np.linalg.solve(K, vals.reshape(shp[0], -1)).reshape(shp)


def dlr_fit_hybridization(rf, it, beta, delta_vals):
    """Plain DLR representation of Delta (``hyb_comp=False`` path, ``block_sparse_solver.py:171-176``):
    poles = DLR frequencies / beta, coefficients = DLR coefficients of Delta."""
    coeffs = vals2coefs(rf, it, np.asarray(delta_vals, dtype=np.complex128))
    return np.asarray(rf, dtype=float) / beta, coeffs


def bethe_delta(beta, it, t_hop=1.0, D=2.0, nquad=4000):
    """t^2 G_bethe(tau) for a semicircular density of states of half-bandwidth D, at the DLR nodes.
    G_bethe(tau) = int rho(e) K(tau/beta, beta e) de, by Gauss-Chebyshev quadrature of the second kind."""
    k = np.arange(1, nquad + 1)
    x = np.cos(k * np.pi / (nquad + 1))
    w = np.pi / (nquad + 1) * np.sin(k * np.pi / (nquad + 1)) ** 2
    # rho(e) de = (2 / (pi D^2)) sqrt(D^2 - e^2) de; with e = D x: (2/pi) sqrt(1 - x^2) dx
    e = D * x
    wt = (2.0 / np.pi) * w
    K = kernel(np.asarray(it)[:, None], beta * e[None, :])
    return t_hop ** 2 * (K @ wt)


def _finish(name, beta, lam, eps, n, ad, rf, it, delta_vals=None, poles=None, coeffs=None, extra=None):
    labels, Fi, Fb, Fdi, Fdb = get_operators(ad)
    dims = np.array(ad.get_subspace_dims(), dtype=np.int32)
    G0, eta0 = atomic_pseudo_particle_greens_function(ad, beta, beta * rel2abs(it))
    if delta_vals is not None:
        poles, coeffs = dlr_fit_hybridization(rf, it, beta, delta_vals)
    return Model(name, beta, lam, eps, n, ad, dims, labels, Fi, Fb, Fdi, Fdb, np.asarray(rf, float), np.asarray(it, float),
                 G0, eta0, np.asarray(poles, float), np.asarray(coeffs, np.complex128), extra or {})


def spin_qn(n_orb):
    """(N_up, N_dn) quantum numbers of every Fock state, orbitals ordered up block then down block."""
    dim = 1 << (2 * n_orb)
    nup = np.array([bin(s & ((1 << n_orb) - 1)).count("1") for s in range(dim)])
    ndn = np.array([bin(s >> n_orb).count("1") for s in range(dim)])
    return [nup, ndn]


def kanamori_hamiltonian(n_orb, U, J, mu, Up=None):
    """Kanamori interaction with spin-flip and pair-hopping terms minus mu N; U' = U - 2J by default."""
    fs = FockSpace(2 * n_orb)
    Up = U - 2 * J if Up is None else Up
    c = [fs.c(k) for k in range(2 * n_orb)]
    cd = [m.T for m in c]
    nn = [cd[k] @ c[k] for k in range(2 * n_orb)]
    up = lambda a: a
    dn = lambda a: n_orb + a
    H = np.zeros((fs.dim, fs.dim))
    for a in range(n_orb):
        H += U * nn[up(a)] @ nn[dn(a)]
    for a, b in itertools.permutations(range(n_orb), 2):
        H += Up * nn[up(a)] @ nn[dn(b)]
        if a < b:
            H += (Up - J) * (nn[up(a)] @ nn[up(b)] + nn[dn(a)] @ nn[dn(b)])
        H += -J * cd[up(a)] @ c[dn(a)] @ cd[dn(b)] @ c[up(b)]
        H += J * cd[up(a)] @ cd[dn(a)] @ c[dn(b)] @ c[up(b)]
    H -= mu * sum(nn)
    return H


def kanamori_half_filling_mu(n_orb, U, J):
    Up = U - 2 * J
    return 0.5 * (U + (n_orb - 1) * Up + (n_orb - 1) * (Up - J))


def one_fermion(rf, it, beta, lam, eps, hyb_pole=0.0):
    """H = 0 spinless fermion with a one-pole hybridization of unit weight
    (``one_fermion_model_helper``, ``test/c++/block_sparse_utils.cpp:17-42``)."""
    fs = FockSpace(1)
    ad = AtomDiag(0 * fs.n_op(0), 1, quantum_numbers=[np.diag(fs.n_op(0))])
    return _finish("one_fermion", beta, lam, eps, 1, ad, rf, it, poles=np.array([hyb_pole]), coeffs=np.ones((1, 1, 1)))


def two_fermion(rf, it, beta, lam, eps, U=3.0, mu=0.0, hyb_pole=-1.5):
    """H = -mu (n0 + n1) + U n0 n1 with N conserved and hyb_coeffs = identity on one pole
    (``two_fermion_model_helper``, ``test/c++/block_sparse_utils.cpp:44-77``)."""
    fs = FockSpace(2)
    n0, n1 = fs.n_op(0), fs.n_op(1)
    H = -mu * (n0 + n1) + U * n0 @ n1
    ad = AtomDiag(H, 2, quantum_numbers=[np.diag(n0 + n1)])
    return _finish("two_fermion", beta, lam, eps, 2, ad, rf, it, poles=np.array([hyb_pole]), coeffs=np.eye(2)[None].astype(complex))


def anderson(rf, it, beta=10.0, lam=100.0, eps=1e-10, U=2.0, mu=1.0):
    """Single-orbital Anderson impurity, (N_up, N_dn) blocks, Bethe hybridization t = 1."""
    fs = FockSpace(2)
    n0, n1 = fs.n_op(0), fs.n_op(1)
    H = U * n0 @ n1 - mu * (n0 + n1)
    ad = AtomDiag(H, 2, quantum_numbers=spin_qn(1))
    d = bethe_delta(beta, it)
    delta = np.zeros((len(it), 2, 2), np.complex128)
    delta[:, 0, 0] = d
    delta[:, 1, 1] = d
    return _finish("anderson_1orb", beta, lam, eps, 2, ad, rf, it, delta_vals=delta)


def kanamori_diag_bethe(rf, it, n_orb, beta, lam, eps, U, J, name):
    mu = kanamori_half_filling_mu(n_orb, U, J)
    H = kanamori_hamiltonian(n_orb, U, J, mu)
    ad = AtomDiag(H, 2 * n_orb, quantum_numbers=spin_qn(n_orb))
    d = bethe_delta(beta, it)
    delta = np.zeros((len(it), 2 * n_orb, 2 * n_orb), np.complex128)
    for i in range(2 * n_orb):
        delta[:, i, i] = d
    return _finish(name, beta, lam, eps, 2 * n_orb, ad, rf, it, delta_vals=delta, extra={"mu": mu, "U": U, "J": J})


def kanamori_2orb(rf, it, beta=20.0, lam=200.0, eps=1e-12):
    """Two-orbital Hubbard-Kanamori at half filling: U = 4, J = 0.5, U' = 3, mu = 4.75."""
    return kanamori_diag_bethe(rf, it, 2, beta, lam, eps, 4.0, 0.5, "kanamori_2orb")


def t2g_3orb(rf, it, beta=50.0, lam=500.0, eps=1e-10, U=3.0, J=0.3, seed=1, n_bath=8):
    """Three-orbital t2g Kanamori (U = 3, J = 0.3, mu = 6.0) with an orbital-off-diagonal,
    spin-diagonal hybridization Delta(tau) = sum_k V_k V_k^T (K(tau/beta, beta w_k)),
    w_k ~ U(-2, 2), V_k ~ N(0, 0.3^2) 3-vectors replicated on both spins (numpy default_rng(seed))."""
    rng = np.random.default_rng(seed)
    w = rng.uniform(-2.0, 2.0, n_bath)
    V = rng.normal(0.0, 0.3, (n_bath, 3))
    mu = kanamori_half_filling_mu(3, U, J)
    H = kanamori_hamiltonian(3, U, J, mu)
    ad = AtomDiag(H, 6, quantum_numbers=spin_qn(3))
    delta = np.zeros((len(it), 6, 6), np.complex128)
    for k in range(n_bath):
        kt = kernel(np.asarray(it), beta * w[k])
        vv = np.outer(V[k], V[k])
        for s in range(2):
            delta[:, 3 * s:3 * s + 3, 3 * s:3 * s + 3] += kt[:, None, None] * vv[None]
    return _finish("t2g_3orb", beta, lam, eps, 6, ad, rf, it, delta_vals=delta,
                   extra={"mu": mu, "bath_w": w, "bath_V": V, "delta": delta})


def seeded_G(model, seed=0):
    """Fixed seeded pseudo-particle propagator: per block, in block order, for l in 0..r-1,
    A_l ~ N(0, 1/r) (d x d), c_l = A_l A_l^T and G_b(tau_i) = sum_l K(tau_i, w_l) c_l."""
    rng = np.random.default_rng(seed)
    r = model.r
    K = kernel(model.it[:, None], model.rf[None, :])
    G = []
    for d in model.dims:
        c = np.empty((r, d, d))
        for l in range(r):
            A = rng.normal(0.0, np.sqrt(1.0 / r), (d, d))
            c[l] = A @ A.T
        G.append(np.einsum("il,lab->iab", K, c).astype(np.complex128))
    return G


def wigner_3j(j1, j2, j3, m1, m2, m3):
    """Wigner 3j symbol of integer arguments (Racah's formula)."""
    from math import factorial, sqrt
    if m1 + m2 + m3 != 0 or abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.0
    if j3 < abs(j1 - j2) or j3 > j1 + j2:
        return 0.0
    f = factorial
    tri = f(j1 + j2 - j3) * f(j1 - j2 + j3) * f(-j1 + j2 + j3) / f(j1 + j2 + j3 + 1)
    pre = sqrt(tri * f(j1 + m1) * f(j1 - m1) * f(j2 + m2) * f(j2 - m2) * f(j3 + m3) * f(j3 - m3))
    s = 0.0
    for t in range(0, j1 + j2 + j3 + 1):
        den = [t, j3 - j2 + t + m1, j3 - j1 + t - m2, j1 + j2 - j3 - t, j1 - t - m1, j2 - t + m2]
        if min(den) < 0:
            continue
        s += (-1) ** t / np.prod([float(f(x)) for x in den])
    return (-1) ** (j1 - j2 - m3) * pre * s


def slater_u_matrix(l, radial_integrals):
    """Slater-Condon interaction U[m1, m2, m3, m4] in the spherical-harmonic basis (m = -l..l):
    sum_k F^k (2l+1)^2 (l k l; 0 0 0)^2 sum_q (-1)^(m1+q+m2) (l k l; -m1 q m3) (l k l; -m2 -q m4), k = 0, 2, .., 2l."""
    n = 2 * l + 1
    U = np.zeros((n, n, n, n))
    ms = range(-l, l + 1)
    for ik, Fk in enumerate(radial_integrals):
        k = 2 * ik
        w0 = (2 * l + 1) ** 2 * wigner_3j(l, k, l, 0, 0, 0) ** 2
        if w0 == 0.0:
            continue
        for a1, m1 in enumerate(ms):
            for a2, m2 in enumerate(ms):
                for a3, m3 in enumerate(ms):
                    for a4, m4 in enumerate(ms):
                        s = 0.0
                        for q in range(-k, k + 1):
                            s += (-1) ** (m1 + q + m2) * wigner_3j(l, k, l, -m1, q, m3) * wigner_3j(l, k, l, -m2, -q, m4)
                        U[a1, a2, a3, a4] += Fk * w0 * s
    return U


def slater_hamiltonian(n_orb, U, mu):
    """H = 1/2 sum_{s1 s2} sum U[a1, a2, a3, a4] c^dag_{s1 a1} c^dag_{s2 a2} c_{s2 a4} c_{s1 a3} - mu N as a dense
    Fock-space matrix (orbital index s * n_orb + a), built by applying the operators to every basis state."""
    n = 2 * n_orb
    dim = 1 << n
    states = np.arange(dim, dtype=np.int64)

    def apply(k, dag, st, sign):
        bit = np.int64(1) << k
        occ = (st & bit) != 0
        ok = ~occ if dag else occ
        below = st & (bit - 1)
        par = np.array([bin(int(x)).count("1") & 1 for x in below]) if len(below) else np.zeros(0, int)
        sign = np.where(ok, sign * np.where(par == 1, -1.0, 1.0), 0.0)
        return st ^ bit, sign

    H = np.zeros((dim, dim))
    nz = np.argwhere(np.abs(U) > 1e-14)
    for s1 in range(2):
        for s2 in range(2):
            for a1, a2, a3, a4 in nz:
                st, sg = states, np.ones(dim)
                st, sg = apply(s1 * n_orb + a3, False, st, sg)
                st, sg = apply(s2 * n_orb + a4, False, st, sg)
                st, sg = apply(s2 * n_orb + a2, True, st, sg)
                st, sg = apply(s1 * n_orb + a1, True, st, sg)
                keep = sg != 0.0
                np.add.at(H, (st[keep], states[keep]), 0.5 * U[a1, a2, a3, a4] * sg[keep])
    H -= mu * np.diag([bin(s).count("1") for s in range(dim)]).astype(float)
    return H


def dshell_5orb(rf, it, beta=20.0, lam=200.0, eps=1e-8, F0=4.0, J=0.7, F4_over_F2=0.625, n_min=4, n_max=6):
    """Five-orbital d shell with the Slater-Condon interaction (F0, and F2, F4 with F2 + F4 = 14 J and F4 / F2 =
    0.625), mu at half filling mu = (45 F0 - 70/49 F2 - 630/441 F4) / 10
    (benchmarks/slater_condon/slater_condon_interaction.py:29), restricted to N = 4..6 (672 states, 16 (N_up, N_dn)
    blocks up to 100 x 100), diagonal Bethe hybridization t = 1."""
    F2 = 14.0 * J / (1.0 + F4_over_F2)
    F4 = F4_over_F2 * F2
    mu = (45 * F0 - 70 / 49 * F2 - 630 / 441 * F4) / 10.0
    U = slater_u_matrix(2, [F0, F2, F4])
    H = slater_hamiltonian(5, U, mu)
    ad = AtomDiag(H, 10, quantum_numbers=spin_qn(5), restrict=lambda s: n_min <= bin(s).count("1") <= n_max)
    d = bethe_delta(beta, it)
    delta = np.zeros((len(it), 10, 10), np.complex128)
    for i in range(10):
        delta[:, i, i] = d
    return _finish("dshell_5orb", beta, lam, eps, 10, ad, rf, it, delta_vals=delta, extra={"mu": mu, "F": (F0, F2, F4)})
