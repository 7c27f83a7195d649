"""numpy model of the sharded evaluation (test infrastructure).

One shard of ``n_shards`` evaluates the partition the CUDA engine uses
(engine.cu ``form_fock`` with ``uw12c_set_shard`` / ``uw12c_set_allreduce``):

* aux functions, dealt out in contiguous balanced ranges ``part(M)``:
  the fitted densities X_D of WV (partial J3_0[:, A]^T d, summed over the
  shards), the 2-el Fock (J3_0[:, A] u, partial), the MO transforms of W, V
  and WV (B1 = H[:, A] P2[A, :] and the stacked RI rows, partial products
  summed over the shards; S^-1 Wst over the shard's aux columns, gathered by
  the same sum) and the t~ dX Fock term (W's aux functions);
* occupied orbitals, ``part(n)``: X_AB and t (partial sums over rows of
  orbitals j / k, summed over the shards), the direct Fock, the same-spin
  three-electron energy and Fock (orbital k of the (j, k) pairs);
* shard 0: the energies built from the summed intermediates (E2d, E2i, E3d,
  E4d) and the same-spin 2-el and 4-el Fock and energies.

``allreduce(array)`` sums an array over the shards in place (the collective
of the caller: gloo ranks on CPU, NCCL on GPUs).  The partial energies and
Fock matrices of all shards sum to ``schedule_model.form_fock``.
"""
import numpy as np

from oracle import uw12_oracle as O
from tests.schedule_model import T3, sq_all


def part(total, shard, n_shards):
    return total * shard // n_shards, total * (shard + 1) // n_shards


def _h1(J3_0, C, lo, hi):
    """H[mu + N k, A] = sum_nu sq(J3_0[:, A])[mu, nu] C[nu, k] for A in [lo, hi)."""
    N, o = C.shape
    sq = sq_all(J3_0[:, lo:hi])
    return np.einsum('mnA,nk->mkA', sq, C).reshape(N * o, hi - lo, order='F')


def _h2(J3ri, C, R, lo, hi):
    N, a = C.shape
    M = J3ri.shape[1]
    J = J3ri.reshape((R, N, M), order='F')[:, :, lo:hi]
    return np.einsum('rmA,mi->riA', J, C).reshape(R * a, hi - lo, order='F')


def form_fock_shard(W, V, WV, Sinv, orbitals, occ, n_active, indirect, s_os, s_ss,
                    shard, n_shards, allreduce):
    """This shard's partial energy terms (dict) and Fock matrices (before the
    final symmetrisation, which is linear and applied after the sum)."""
    n_spin = len(orbitals)
    Co = O.occupation_weighted_orbitals(orbitals, occ)
    Ca = O.freeze_core(Co, n_active)
    N, R = W.n_ao, W.n_ri
    Rp = N + R
    pt = lambda total: part(total, shard, n_shards)
    lead = shard == 0
    f = lambda s, sp: O.get_energy_spin_factor(n_spin, s, sp, s_os, s_ss)
    half = 0.5 if n_spin == 1 else 1.0
    two = 2 if n_spin == 1 else 1
    do_ind = indirect and s_ss != 0
    F = [np.zeros((N, N)) for _ in range(n_spin)]
    E = {k: 0.0 for k in ('2d', '2i', '3d', '4d', '4i', '3i')}

    # ---- 2-el: fitted densities and Fock over this shard's aux range of WV
    MX = WV.n_df
    lam = WV.df_vals
    xlo, xhi = pt(MX)
    XDr = np.zeros((MX, n_spin))
    for s in range(n_spin):
        d = O.lower(two * Ca[s] @ Ca[s].T, 2.0)
        XDr[xlo:xhi, s] = WV.J3_0[:, xlo:xhi].T @ d
    allreduce(XDr)
    XD = 0.5 * n_spin * (WV.P2.T @ XDr)
    for s in range(n_spin):
        vc = np.zeros(MX)
        for sp in range(n_spin):
            ff = f(s, sp)
            if ff == 0:
                continue
            if lead:
                E['2d'] += 0.5 * ff * XD[:, s] @ (lam * XD[:, sp])
            vc += 0.5 * n_spin * ff * lam * XD[:, sp]
        u = WV.P2 @ vc
        F[s] += O.square(WV.J3_0[:, xlo:xhi] @ u[xlo:xhi])
    if do_ind:
        for s in range(n_spin):
            a = Ca[s].shape[1]
            if a == 0:
                continue
            B1 = _h1(WV.J3_0, Ca[s], xlo, xhi) @ WV.P2[xlo:xhi, :]
            allreduce(B1)
            if not lead:
                continue
            B2 = T3(B1, Ca[s])
            E['2i'] += -0.5 * two * s_ss * np.sum(B2 * B2 * lam[None, :])
            r1 = B1.reshape(N, a * MX, order='F')
            r1l = (B1 * lam[None, :]).reshape(N, a * MX, order='F')
            F[s] += -s_ss * (r1 @ r1l.T)

    # ---- MO transforms over this shard's aux range of W and V, summed
    B1 = {}; B2 = {}; Wp = {}; SVp = {}
    for s in range(n_spin):
        o = Co[s].shape[1]; a = Ca[s].shape[1]; c = o - a
        for X, nm in ((W, 'W'), (V, 'V')):
            M = X.n_df
            lo, hi = pt(M)
            b1 = _h1(X.J3_0, Co[s], lo, hi) @ X.P2[lo:hi, :]
            allreduce(b1)
            B1[nm, s] = b1
            B2[nm, s] = T3(b1, Ca[s])
            st3 = np.zeros((Rp, a, M))
            st3[N:] = (_h2(X.J3_ri_0, Ca[s], R, lo, hi) @ X.P2[lo:hi, :]).reshape(
                (R, a, M), order='F')
            st = st3.reshape((Rp * a, M), order='F')
            allreduce(st)
            st3 = st.reshape((Rp, a, M), order='F')
            st3[:N] = b1.reshape((N, o, M), order='F')[:, c:, :]
            Wp[nm, s] = st3.reshape((Rp * a, M), order='F')
            # S^-1 Wst over this shard's aux columns, gathered by the sum
            sv = np.zeros((Rp, a * M))
            sv[:, a * lo:a * hi] = Sinv @ Wp[nm, s].reshape(Rp, a * M, order='F')[:, a * lo:a * hi]
            allreduce(sv)
            SVp[nm, s] = sv.reshape(Rp * a, M, order='F')

    # ---- X_AB and t over this shard's orbitals, summed
    lw, lv = W.df_vals, V.df_vals
    Xab, tab = [], []
    for s in range(n_spin):
        o = Co[s].shape[1]; a = Ca[s].shape[1]
        jlo, jhi = pt(a)
        klo, khi = pt(o)
        x = Wp['W', s][Rp * jlo:Rp * jhi].T @ SVp['V', s][Rp * jlo:Rp * jhi]
        t = B2['W', s][a * klo:a * khi].T @ B2['V', s][a * klo:a * khi]
        allreduce(x)
        allreduce(t)
        Xab.append(x); tab.append(t)
    tt = [lw[:, None] * tab[s] * lv[None, :] for s in range(n_spin)]
    if lead:
        for s in range(n_spin):
            for sp in range(n_spin):
                ff = f(s, sp)
                E['3d'] -= ff * np.sum(Xab[s] * tt[sp])
                if ff != 0:
                    E['4d'] += 0.5 * ff * np.sum(tt[sp] * tab[s])

    # ---- direct Fock over this shard's occupied orbitals
    kap4 = 2 * half
    for s in range(n_spin):
        o = Co[s].shape[1]; a = Ca[s].shape[1]; c = o - a
        klo, khi = pt(o)
        if khi == klo:
            continue
        T4 = sum(f(s, sp) * tt[sp] for sp in range(n_spin))
        Xc = sum(half * f(s, sp) * Xab[sp] for sp in range(n_spin))
        Y = (kap4 if a == 0 else 0.5 * kap4) * T4 - lw[:, None] * Xc * lv[None, :]
        MW = W.n_df
        bw = B1['W', s].reshape((N, o, MW), order='F')[:, klo:khi, :]
        bv = B1['V', s].reshape((N, o, V.n_df), order='F')[:, klo:khi, :]
        Z3 = np.einsum('mkA,AB->mkB', bw, Y)
        for k in range(klo, khi):
            if a > 0 and k >= c:
                Z3[:, k - klo, :] *= 2.0
        F[s] += np.einsum('mkB,nkB->mn', Z3, bv)

    # ---- t~ dX over this shard's range of W's aux functions
    for sp in range(n_spin):
        Tc = sum(half * f(s, sp) * tt[s] for s in range(n_spin))
        T2m = W.P2 @ Tc @ V.P2.T
        alo, ahi = pt(W.n_df)
        sm = V.J3_0 @ T2m[alo:ahi, :].T
        pm = V.J3_ri_0 @ T2m[alo:ahi, :].T
        H = np.zeros((Rp, N, ahi - alo))
        H[:N] = sq_all(sm)
        H[N:] = pm.reshape((R, N, ahi - alo), order='F')
        U = np.einsum('pq,qnA->pnA', Sinv, H)
        G = np.zeros((Rp, N, ahi - alo))
        G[:N] = sq_all(W.J3_0[:, alo:ahi])
        G[N:] = W.J3_ri_0[:, alo:ahi].reshape((R, N, ahi - alo), order='F')
        F[sp] += -np.einsum('pmA,pnA->mn', G, U)

    # ---- same-spin terms: 4-el on shard 0, 3-el over this shard's k
    if do_ind:
        for s in range(n_spin):
            o = Co[s].shape[1]; a = Ca[s].shape[1]; c = o - a
            if a == 0 or o == 0:
                continue
            klo, khi = pt(o)
            b2wl = B2['W', s] * lw[None, :]; b2vl = B2['V', s] * lv[None, :]
            if lead:
                W4 = (b2wl @ B2['W', s].T).reshape((a, o, a, o), order='F')
                V4 = (b2vl @ B2['V', s].T).reshape((a, o, a, o), order='F')
                E['4i'] += -0.5 * two * s_ss * np.einsum('iljk,ikjl->', W4, V4)
                W43 = ((B1['W', s] * lw[None, :]) @ B2['W', s].T).reshape((N, o, a, o), order='F')
                V43 = ((B1['V', s] * lv[None, :]) @ B2['V', s].T).reshape((N, o, a, o), order='F')
                Fi = -2 * np.einsum('mijk,njik->mn', W43[:, c:], V43[:, c:])
                if c > 0:
                    Ff = -2 * np.einsum('mljk,nkjl->mn', W43, V43)
                    Fi = 0.5 * (Fi + Ff)
                F[s] += s_ss * Fi
            # 3-el energy: pairs (j, k) with k in [klo, khi)
            YW = (Wp['W', s] @ b2wl.T).reshape((Rp, a, a, o), order='F')
            ZV = (SVp['V', s] @ b2vl.T).reshape((Rp, a, a, o), order='F')
            E['3i'] += two * s_ss * np.einsum('pijk,pjik->', YW[..., klo:khi], ZV[..., klo:khi])
            Fk = np.zeros((N, N))
            for (Xn, Yn, Xi, Yi) in (('W', 'V', W, V), ('V', 'W', V, W)):
                lx = Xi.df_vals; ly = Yi.df_vals
                ZY = (SVp[Yn, s] @ (B1[Yn, s] * ly[None, :]).T).reshape((Rp, a, N, o), order='F')
                xh = Xi.P2 @ (lx[:, None] * B2[Xn, s].T)
                gao = sq_all(Xi.J3_0 @ xh)
                gri = (Xi.J3_ri_0 @ xh).reshape((R, N, a * o), order='F')
                G = np.concatenate([gao, gri], axis=0).reshape((Rp, N, a, o), order='F')
                Fk += np.einsum('pajk,pjbk->ab', G[..., klo:khi], ZY[..., klo:khi])
            # k-term: active orbitals c + i inside [klo, khi)
            ilo, ihi = max(klo, c) - c, khi - c
            if ihi > ilo:
                b1w = (B1['W', s] * lw[None, :]).reshape((N, o, W.n_df), order='F')[:, c:, :]
                Wk = (Wp['W', s] @ b1w.reshape(N * a, W.n_df, order='F').T).reshape(
                    (Rp, a, N, a), order='F')
                ZYV = (SVp['V', s] @ (B1['V', s] * lv[None, :]).T).reshape((Rp, a, N, o),
                                                                           order='F')
                Fk += np.einsum('pibj,pjai->ba', Wk[:, ilo:ihi], ZYV[:, :, :, c + ilo:c + ihi])
            F[s] += s_ss * Fk
    return E, F
