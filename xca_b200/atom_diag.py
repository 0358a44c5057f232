"""Host-side Fock-space builder: a minimal stand-in for TRIQS ``atom_diag`` plus the reference's
``get_operators`` / atomic-propagator set-up.

This is set-up code that runs once per model on the host (numpy), as in the reference, where it is
C++/Python host code:

* ``get_operators_impl``     ``c++/triqs_xca/atom_diag_utils.cpp:39-185``  (symmetry sets, F / F^dag blocks)
* ``H_to_atom_prop_blocks``  ``c++/triqs_xca/atom_diag_utils.cpp:276-315``
* ``atomic_pseudo_particle_greens_function``  ``python/triqs_xca/block_sparse_solver.py:1305-1328``

Fock state ``s`` has bit ``k`` set when fundamental operator ``k`` is occupied; the fermion sign of
``c_k`` is ``(-1)^popcount(s & ((1 << k) - 1))``, the convention pinned by
``test/c++/test_atom_diag_utils.cpp:99-118``.  Subspaces are listed by particle number, then by their
smallest Fock state, and the Fock states of a subspace ascend: the ordering the same test pins for
its Hamiltonian blocks (:205-221).
"""

import numpy as np


def popcount(x):
    return bin(int(x)).count("1")


class FockSpace:
    """Dense matrices of c_k and c^dag_k on the 2^n Fock states of n fundamental operators."""

    def __init__(self, n):
        self.n = n
        self.dim = 1 << n

    def c(self, k):
        m = np.zeros((self.dim, self.dim))
        for s in range(self.dim):
            if s & (1 << k):
                t = s ^ (1 << k)
                m[t, s] = -1.0 if popcount(s & ((1 << k) - 1)) % 2 else 1.0
        return m

    def cdag(self, k):
        return self.c(k).T.copy()

    def n_op(self, k):
        return np.diag([(s >> k) & 1 for s in range(self.dim)]).astype(float)


class AtomDiag:
    """Block-diagonalisation of a local Hamiltonian in Fock-space subspaces.

    ``H`` is the dense (2^n x 2^n) Hamiltonian.  ``quantum_numbers`` is either ``None`` (automatic
    partition: connected components of H, then merged until every c_k and c^dag_k maps each
    subspace into a single subspace, the rule of TRIQS' autopartition) or a list of length-2^n
    arrays of diagonal quantum numbers (for example N_up and N_dn).  ``restrict`` optionally keeps
    only Fock states for which it returns True (used for the N = 4..6 d-shell model).
    """

    def __init__(self, H, n, quantum_numbers=None, restrict=None, subspaces=None):
        H = np.asarray(H)
        self.H = H
        self.n = n
        self.fock = FockSpace(n)
        dim = 1 << n
        self.full_hilbert_space_dim = dim
        keep = [s for s in range(dim) if restrict is None or restrict(s)]
        self.c_full = [self.fock.c(k) for k in range(n)]
        self.cdag_full = [self.fock.cdag(k) for k in range(n)]
        if subspaces is not None:
            # an explicit partition (as saved by to_dict): lists of Fock states
            subspaces = [[int(x) for x in sub] for sub in subspaces]
            keep = sorted(x for sub in subspaces for x in sub)
        elif quantum_numbers is not None:
            qn = [np.asarray(q) for q in quantum_numbers]
            groups = {}
            order = []
            for s in keep:
                key = tuple(float(q[s]) for q in qn)
                if key not in groups:
                    groups[key] = []
                    order.append(key)
                groups[key].append(s)
            subspaces = [groups[k] for k in order]
        else:
            subspaces = self._autopartition(H, keep)
        self.fock_states = [np.array(sorted(s), dtype=np.int64) for s in subspaces]
        self.fock_states.sort(key=lambda a: (popcount(a[0]), a[0]))
        self.n_subspaces = len(self.fock_states)
        self._state_sub = {}
        for i, fs in enumerate(self.fock_states):
            for s in fs:
                self._state_sub[int(s)] = i
        # Hamiltonian blocks and their diagonalisation
        self.H_blocks = [H[np.ix_(fs, fs)] for fs in self.fock_states]
        if self.H_blocks and max(np.max(np.abs(H[np.ix_(a, b)])) for i, a in enumerate(self.fock_states)
                                 for j, b in enumerate(self.fock_states) if i != j) > 1e-12:
            raise ValueError("AtomDiag: H is not block diagonal in the requested subspaces")
        evals, evecs = [], []
        for h in self.H_blocks:
            e, u = np.linalg.eigh(h)
            evals.append(e)
            evecs.append(u)
        self.gs_energy = min(float(np.min(e)) for e in evals)
        self.energies = [e - self.gs_energy for e in evals]
        self.unitary_matrices = evecs
        # connections
        self.c_connection = np.full((n, self.n_subspaces), -1, dtype=np.int64)
        self.cdag_connection = np.full((n, self.n_subspaces), -1, dtype=np.int64)
        for k in range(n):
            for s, fs in enumerate(self.fock_states):
                for mats, conn in ((self.c_full, self.c_connection), (self.cdag_full, self.cdag_connection)):
                    tgt = set()
                    sub = mats[k][:, fs]
                    rows = np.nonzero(np.any(np.abs(sub) > 0, axis=1))[0]
                    for row in rows:
                        if int(row) in self._state_sub:
                            tgt.add(self._state_sub[int(row)])
                    if len(tgt) > 1:
                        raise ValueError("AtomDiag: an operator maps one subspace into several")
                    if tgt:
                        conn[k, s] = tgt.pop()

    def _autopartition(self, H, keep):
        parent = {s: s for s in keep}

        def find(x):
            while parent[x] != x:
                parent[x] = parent[parent[x]]
                x = parent[x]
            return x

        def union(a, b):
            ra, rb = find(a), find(b)
            if ra != rb:
                parent[max(ra, rb)] = min(ra, rb)

        kset = set(keep)
        for a in keep:
            for b in np.nonzero(np.abs(H[a]) > 0)[0]:
                if int(b) in kset:
                    union(a, int(b))
        changed = True
        while changed:
            changed = False
            for mats in (self.c_full, self.cdag_full):
                for mk in mats:
                    image = {}
                    for s in keep:
                        rows = np.nonzero(mk[:, s])[0]
                        for row in rows:
                            row = int(row)
                            if row not in kset:
                                continue
                            root = find(s)
                            if root in image and find(image[root]) != find(row):
                                union(image[root], row)
                                changed = True
                            image.setdefault(root, row)
        groups = {}
        for s in keep:
            groups.setdefault(find(s), []).append(s)
        return list(groups.values())

    def to_dict(self):
        """The Hamiltonian and the subspace partition, from which ``from_dict`` rebuilds this object."""
        return {"H": self.H, "n": self.n, "subspaces": [fs.copy() for fs in self.fock_states]}

    @classmethod
    def from_dict(cls, d):
        return cls(d["H"], int(d["n"]), subspaces=d["subspaces"])

    def get_subspace_dims(self):
        return [len(fs) for fs in self.fock_states]

    def get_op_mat(self, op):
        """Block form of a Fock-space operator ``op`` (a dense 2^n x 2^n matrix, e.g. built from
        ``FockSpace.c`` / ``n_op``): per subspace b the subspace it maps b to (-1 if none) and the
        (d_target x d_b) block in the Fock basis.  These are the blocks that the reference builds from
        ``ad.get_op_mat(op)`` and the unitary matrices (``setup_ops_from_triqs_2nd_quant_ops``,
        ``c++/triqs_xca/block_sparse_backbone.cpp:810-840``; ``expectation_value``,
        ``c++/triqs_xca/block_sparse.cpp:803-811``): the basis of G and of the field operators here."""
        op = np.asarray(op)
        nb = self.n_subspaces
        index = np.full(nb, -1, dtype=np.int32)
        blocks = [None] * nb
        for b, fi in enumerate(self.fock_states):
            sub = op[:, fi]
            rows = np.nonzero(np.any(np.abs(sub) > 0, axis=1))[0]
            tgt = {self._state_sub[int(x)] for x in rows if int(x) in self._state_sub}
            if len(tgt) > 1:
                raise ValueError("AtomDiag.get_op_mat: the operator maps a subspace into several subspaces")
            if not tgt:
                continue
            t = tgt.pop()
            index[b] = t
            blocks[b] = np.asarray(op[np.ix_(self.fock_states[t], fi)], dtype=np.complex128)
        return index, blocks


def get_operators(ad, n=None):
    """Symmetry sets and per-block F / F^dag slabs (``atom_diag_utils.cpp:39-185``).

    Returns ``(sym_set_labels, F_index, F_blocks, Fd_index, Fd_blocks)`` where ``F_index[s, b]`` is
    the target subspace of set ``s`` acting on block ``b`` (-1 if none) and ``F_blocks[s][b]`` has
    shape ``(q_s, d_target, d_b)`` in the Fock basis.
    """
    n = ad.n if n is None else n
    labels = np.zeros(n, dtype=np.int64)
    counter = 0
    for o in range(n):
        for o2 in range(o):
            if np.array_equal(ad.c_connection[o], ad.c_connection[o2]):
                labels[o] = labels[o2]
                break
        else:
            labels[o] = counter
            counter += 1
    nq = counter
    nb = ad.n_subspaces
    F_index = np.full((nq, nb), -1, dtype=np.int32)
    Fd_index = np.full((nq, nb), -1, dtype=np.int32)
    F_blocks = [[None] * nb for _ in range(nq)]
    Fd_blocks = [[None] * nb for _ in range(nq)]
    members = [[o for o in range(n) if labels[o] == s] for s in range(nq)]
    for s in range(nq):
        rep = members[s][0]
        for b in range(nb):
            for conn, index, blocks, mats in ((ad.c_connection, F_index, F_blocks, ad.c_full),
                                              (ad.cdag_connection, Fd_index, Fd_blocks, ad.cdag_full)):
                tgt = int(conn[rep, b])
                if tgt < 0:
                    continue
                index[s, b] = tgt
                fi, ff = ad.fock_states[b], ad.fock_states[tgt]
                blocks[s][b] = np.stack([mats[o][np.ix_(ff, fi)] for o in members[s]]).astype(np.complex128)
    return labels, F_index, F_blocks, Fd_index, Fd_blocks


def atomic_pseudo_particle_greens_function(ad, beta, tau):
    """``atomic_pseudo_particle_greens_function`` (``block_sparse_solver.py:1305-1328``):
    G_b(tau) = -U_b exp(-tau (E_b - eta0)) U_b^dag with eta0 = -log(Z0) / beta."""
    Z0 = sum(np.sum(np.exp(-beta * E)) for E in ad.energies)
    eta0 = -np.log(Z0) / beta
    tau = np.asarray(tau, dtype=float)
    G = []
    for U, E in zip(ad.unitary_matrices, ad.energies):
        gd = -np.exp(-tau[:, None] * (E - eta0)[None, :])
        G.append(np.einsum("ij,tj,kj->tik", U, gd, np.conj(U)).astype(np.complex128))
    return G, eta0
