"""A CPU shard with the engine's shard interface, computed by the FP64
oracle (test infrastructure): the MTTKRP of its own nonzeros (COO) and the
reference's ALS update steps (adatm_cpd.c:256-373) in numpy."""
import numpy as np

import oracle as O


class OracleShard:
    def __init__(self, inds, vals, dims, R, seed=0):
        self.inds, self.vals, self.dims, self.R = inds, vals, [int(d) for d in dims], R
        self.A = [np.array(m, dtype=np.float64) for m in O.init_factors(self.dims, R, seed)]
        self.N = len(self.dims)

    def ttnorm(self):
        return float(np.sum(self.vals * self.vals))

    def set_ttnorm(self, v):
        self.ttn = v

    def als_begin(self, graph=False):
        self.G = [a.T @ a for a in self.A]
        self.it = 0
        self.lam = np.ones(self.R)

    def mttkrp_into(self, m, buf):
        if self.vals.size:
            M = O.mttkrp_coo(self.inds, self.vals, self.dims, self.A, m, self.R)
        else:
            M = np.zeros((self.dims[m], self.R))
        buf.numpy()[:] = M.reshape(-1)

    def update_from(self, m, buf):
        M = buf.numpy().reshape(self.dims[m], self.R)
        V = np.ones((self.R, self.R))
        for k in range(self.N):
            if k != m:
                V *= self.G[k]
        A = M @ np.linalg.inv(V)
        if self.it == 0:
            lam = np.sqrt(np.sum(A * A, axis=0))
        else:
            lam = np.maximum(np.max(A, axis=0), 1.0)
        A = A / lam
        self.A[m], self.lam = A, lam
        self.G[m] = A.T @ A
        if m == self.N - 1:
            self.inner = float(np.sum(np.sum(A * M, axis=0) * lam))

    def fit_step(self):
        H = np.ones((self.R, self.R))
        for g in self.G:
            H *= g
        norm = abs(float(self.lam @ H @ self.lam))
        self.it += 1
        return 1.0 - np.sqrt(self.ttn + norm - 2.0 * self.inner) / np.sqrt(self.ttn)
