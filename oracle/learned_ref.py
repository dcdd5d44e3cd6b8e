"""CPU oracle of the learned p' preconditioner (test infrastructure only).

A float64 numpy restatement of the network that
axisim-software_b200/csrc/learned.hpp defines and learned.cu trains: the same
levels, channel widths, weight groups, flat parameter layout, input features,
loss and gradient. The reference has no learned preconditioner, so there are no
golden vectors for this part; the oracle's gradient is pinned instead by central
finite differences of its own loss (tests/test_learned_cpu.py), and the CUDA
forward/backward kernels are checked against it (tests/test_gpu_learned.py).

Graph inputs are the multigrid hierarchy as the solvers report it: the level-0
cell graph from the packed mesh, and per level the fine-to-coarse map and the
coarse CSR (axisim_mg_level_maps / Oracle.mg_level_maps).
"""
import numpy as np
import scipy.sparse as sp

CHANNELS = (16, 32, 64)
COARSE_CHANNELS = 128
MAX_LEVELS = 16


def level0_neighbours(mesh):
    """Per-cell neighbour lists of the packed mesh in slot order, as finestLevel
    (csrc/host_prep.cpp) builds them; boundary slots dropped."""
    cfs, cfi = mesh["cellFaceStart"], mesh["cellFaceIDs"]
    own, nb = mesh["faceOwner"], mesh["faceNeighbor"]
    N = int(mesh["nCells"])
    rows = np.repeat(np.arange(N), np.diff(cfs))
    f = cfi
    other = np.where(own[f] == rows, nb[f], np.where(nb[f] == rows, own[f], -1))
    keep = (other >= 0) & (other != rows)
    return N, rows[keep], other[keep]


def hierarchy(mesh, level_maps, n_levels):
    """[(N_l, rows, cols, c2c)] for l < n_levels; level_maps(l) -> (c2c, f2c,
    coarse faceStart, coarse faceNeighbor)."""
    out = []
    N, r, c = level0_neighbours(mesh)
    for l in range(n_levels):
        c2c = level_maps(l)[0] if l + 1 < n_levels else None
        out.append((N, r, c, c2c))
        if c2c is None:
            break
        _, _, cfs, cfn = level_maps(l)
        Nc = len(cfs) - 1
        rows = np.repeat(np.arange(Nc), np.diff(cfs))
        keep = (cfn >= 0) & (cfn != rows)
        N, r, c = Nc, rows[keep], cfn[keep]
    return out


def matrix(mesh, ac, af_slots):
    """Sparse A from its diagonal and the off-diagonals in the mesh's slot
    order (cellFaceStart / cellFaceIDs; boundary slots ignored)."""
    N, r, c = level0_neighbours(mesh)
    cfs, cfi = mesh["cellFaceStart"], mesh["cellFaceIDs"]
    own, nb = mesh["faceOwner"], mesh["faceNeighbor"]
    rows = np.repeat(np.arange(N), np.diff(cfs))
    other = np.where(own[cfi] == rows, nb[cfi], np.where(nb[cfi] == rows, own[cfi], -1))
    keep = (other >= 0) & (other != rows)
    af = np.asarray(af_slots, np.float64)[keep]
    return sp.csr_matrix((np.r_[af, np.asarray(ac, np.float64)], (np.r_[rows[keep], np.arange(N)],
                                                                   np.r_[other[keep], np.arange(N)])), shape=(N, N))


def random_spd_system(mesh, rng):
    """A symmetric, diagonally dominant p'-like matrix on the mesh (negative
    off-diagonals, a random positive surplus on the diagonal), as (A_C, A_F in
    slot order)."""
    N = int(mesh["nCells"])
    F = int(mesh["nFaces"])
    w = rng.uniform(0.5, 2.0, F)
    cfs, cfi = mesh["cellFaceStart"], mesh["cellFaceIDs"]
    nb = mesh["faceNeighbor"]
    af = np.where(nb[cfi] >= 0, -w[cfi], 0.0)
    rows = np.repeat(np.arange(N), np.diff(cfs))
    ac = np.bincount(rows, weights=-af, minlength=N) + rng.uniform(0.01, 0.1, N)
    return ac, af


class NetRef:
    def __init__(self, levels):
        self.L = min(len(levels), MAX_LEVELS)
        lv = levels[:self.L]
        self.N = [x[0] for x in lv]
        self.C = [CHANNELS[l] if l < 3 else COARSE_CHANNELS for l in range(self.L)]
        self.M, self.P, self.U = [], [], []  # neighbour mean, pool from l-1, unpool from l+1
        for N, r, c, _ in lv:
            A = sp.csr_matrix((np.ones(len(r)), (r, c)), shape=(N, N))
            deg = np.asarray(A.sum(1)).ravel()
            self.M.append(sp.diags(np.where(deg > 0, 1.0 / np.maximum(deg, 1), 0.0)) @ A)
        for l in range(self.L):
            if l > 0:
                c2c = lv[l - 1][3]
                Nf, Nc = self.N[l - 1], self.N[l]
                Pm = sp.csr_matrix((np.ones(Nf), (c2c, np.arange(Nf))), shape=(Nc, Nf))
                cnt = np.asarray(Pm.sum(1)).ravel()
                self.P.append(sp.diags(np.where(cnt > 0, 1.0 / np.maximum(cnt, 1), 0.0)) @ Pm)
            else:
                self.P.append(None)
            if l + 1 < self.L:
                self.U.append(sp.csr_matrix((np.ones(self.N[l]), (np.arange(self.N[l]), lv[l][3])),
                                            shape=(self.N[l], self.N[l + 1])))
            else:
                self.U.append(None)
        self._layers()

    def _layers(self):
        """Layer list in forward order; weight groups allocated in first-use
        order, weights [K][Cout] row-major then bias [Cout]."""
        L, C = self.L, self.C
        self.groups = {}
        self.n_params = 0

        def group(key, K, Co):
            if key not in self.groups:
                self.groups[key] = (self.n_params, K, Co)
                self.n_params += K * Co + Co
            return key

        lay = [dict(key=group("in", 2, C[0]), ins=[("feat", "id", None)], add=None, out="H0", relu=True),
               dict(key=group("enc0", 2 * C[0], C[0]), ins=[("H0", "id", 0), ("H0", "nb", 0)], add=None, out="E0",
                    relu=True)]
        for l in range(1, L):
            lay.append(dict(key=group(f"down{min(l, 4)}", C[l - 1], C[l]), ins=[(f"E{l - 1}", "pool", l)], add=None,
                            out=f"H{l}", relu=True))
            lay.append(dict(key=group(f"enc{min(l, 3)}", 2 * C[l], C[l]), ins=[(f"H{l}", "id", l), (f"H{l}", "nb", l)],
                            add=None, out=f"E{l}", relu=True))
        m = L - 1
        lay.append(dict(key=group(f"mid{min(m, 3)}", 2 * C[m], C[m]), ins=[(f"E{m}", "id", m), (f"E{m}", "nb", m)],
                        add=None, out=f"D{m}", relu=True))
        for l in range(L - 2, -1, -1):
            lay.append(dict(key=group(f"up{min(l, 3)}", C[l + 1], C[l]), ins=[(f"D{l + 1}", "unpool", l)],
                            add=f"E{l}", out=f"S{l}", relu=True))
            lay.append(dict(key=group(f"dec{min(l, 3)}", 2 * C[l], C[l]), ins=[(f"S{l}", "id", l), (f"S{l}", "nb", l)],
                            add=None, out=f"D{l}", relu=True))
        lay.append(dict(key=group("out", C[0], 1), ins=[("D0", "id", 0)], add=None, out="Y", relu=False))
        self.layers = lay

    def init_params(self, seed=0):
        rng = np.random.default_rng(seed)
        p = np.zeros(self.n_params)
        for key, (off, K, Co) in self.groups.items():
            a = np.sqrt(3.0 / K) if key == "out" else np.sqrt(6.0 / K)
            p[off:off + K * Co] = rng.uniform(-a, a, K * Co)
        return p

    def _W(self, p, key):
        off, K, Co = self.groups[key]
        return p[off:off + K * Co].reshape(K, Co), p[off + K * Co:off + K * Co + Co]

    def _xf(self, X, kind, l):
        if kind == "id":
            return X
        return {"nb": self.M, "pool": self.P, "unpool": self.U}[kind][l] @ X

    def _xf_adj(self, G, kind, l):
        if kind == "id":
            return G
        return {"nb": self.M, "pool": self.P, "unpool": self.U}[kind][l].T @ G

    @staticmethod
    def features(b, ac, deficit):
        b, ac = np.asarray(b, np.float64), np.asarray(ac, np.float64)
        q = np.where(ac != 0, b / np.where(ac != 0, ac, 1.0), 0.0)
        sigma = np.sqrt(np.mean(q * q))
        x0 = q / sigma if sigma > 0 else np.zeros_like(q)
        return np.stack([x0, np.asarray(deficit, np.float64)], axis=1), sigma

    def forward(self, p, feat):
        T = {"feat": feat}
        Zs = []
        for ly in self.layers:
            Z = np.concatenate([self._xf(T[name], kind, l) for name, kind, l in ly["ins"]], axis=1)
            W, bias = self._W(p, ly["key"])
            Y = Z @ W + bias
            if ly["add"]:
                Y = Y + T[ly["add"]]
            if ly["relu"]:
                Y = np.maximum(Y, 0.0)
            T[ly["out"]] = Y
            Zs.append(Z)
        return T, Zs

    def loss_and_grad(self, p, b, target, ac, deficit, A):
        """Loss 1 - (y.b)^2 / ((y.A y)(b.t)): the energy-norm error left after
        the best scaling of the output y (A t = b), and its gradient in the
        flat layout."""
        feat, _ = self.features(b, ac, deficit)
        T, Zs = self.forward(p, feat)
        y = T["Y"][:, 0]
        b = np.asarray(b, np.float64)
        Ay = A @ y
        c, ey, et = y @ b, y @ Ay, b @ np.asarray(target, np.float64)
        ey = ey if ey > 0 else 1e-300
        et = et if et > 0 else 1.0
        loss = 1.0 - c * c / (ey * et)
        G = {name: np.zeros_like(v) for name, v in T.items()}
        G["Y"] = (-2.0 * c / (ey * et) * b + 2.0 * c * c / (ey * ey * et) * Ay)[:, None]
        grad = np.zeros_like(p)
        for ly, Z in zip(reversed(self.layers), reversed(Zs)):
            g = G[ly["out"]]
            if ly["relu"]:
                g = g * (T[ly["out"]] > 0)
            W, _ = self._W(p, ly["key"])
            off, K, Co = self.groups[ly["key"]]
            grad[off:off + K * Co] += (Z.T @ g).ravel()
            grad[off + K * Co:off + K * Co + Co] += g.sum(0)
            if ly["add"]:
                G[ly["add"]] += g
            dZ = g @ W.T
            o = 0
            for name, kind, l in ly["ins"]:
                cw = T[name].shape[1]
                if name != "feat":
                    G[name] += self._xf_adj(dZ[:, o:o + cw], kind, l)
                o += cw
        return loss, grad

    def predict(self, p, r, ac, deficit):
        feat, sigma = self.features(r, ac, deficit)
        T, _ = self.forward(p, feat)
        return sigma * T["Y"][:, 0]
