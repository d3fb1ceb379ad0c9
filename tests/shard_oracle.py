"""One rank's share of the submatrix step on the CPU oracle, with the four
methods of ptb_b200.distributed.DeviceShard (test infrastructure: it lets the
multi-rank protocol run on gloo ranks without a GPU)."""
import numpy as np

from oracle import ptb_oracle as O


class OracleShard:
    def plan(self, ndim, Hvec, Svec, n, xyz, aoat, columns, mode, partition, opts):
        self.ndim = ndim
        self.H = O.blowsym(ndim, O.filter_matrix_sym(Hvec, opts.filter))
        self.S = O.blowsym(ndim, O.filter_matrix_sym(Svec, opts.filter))
        self.comb = O.submatrix_columns(columns, ndim, aoat, n, partition)
        self.maps = [O.submatrix_map(self.H, self.S, np.asarray(owned)) for owned in self.comb]
        return np.array([len(m) for m in self.maps], dtype=np.int64)

    def prepare(self, ids):
        self.eig = []
        for k in ids:
            mp, owned = self.maps[k], np.asarray(self.comb[k])
            m = len(mp)
            imap = np.full(self.ndim, -1, dtype=np.int64)
            imap[mp] = np.arange(m)
            Hs, Ss = self.H[np.ix_(mp, mp)], self.S[np.ix_(mp, mp)]
            e, U, _ = O.sygvd(Hs, Ss)
            io = imap[owned]
            fe = np.sum((Ss @ U)[io, :] * U[io, :], axis=0)
            self.eig.append((mp, imap, owned, e, U, fe))

    def nel(self, mu):
        v = 0.0
        for (_, _, _, e, _, fe) in self.eig:
            occ = np.where(e < mu, 2.0, np.where(e == mu, 1.0, 0.0))
            v += float(np.sum(fe * occ))
        return v

    def finish(self, ndim, mu):
        P = np.zeros((ndim, ndim))
        for (mp, imap, owned, e, U, _) in self.eig:
            occ = np.where(e < mu, 2.0, np.where(e == mu, 1.0, 0.0))
            P[np.ix_(mp, owned)] = O.dmat(occ, U)[:, imap[owned]]
        return O.packsym(P)
