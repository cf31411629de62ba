"""Batched SCF: many independent molecules of uneven size converged together.

Every iteration runs one batched Fock build (engine.BatchEngine: one launch
per quartet class over all molecules' tasks) and the reference's SCF step
(RestrictedHartreeFock.cpp:61-166, UnrestrictedHartreeFock.cpp:87-191) for
all molecules at once in torch on the device: F = h + G, DIIS (keep 6, start
at 5; DIIS.h:9-96), F' = V F V, batched eigensolve, new density, energy,
mixing, the reference's convergence test per molecule.  Molecules that have
converged drop out of the following builds (the engine's `active` mask), and
once half of the working set has converged the torch state shrinks to the
molecules still iterating (re-padded to the largest of them), so the cost of
a step follows the active count.  Matrices are padded to the largest molecule
of the working set: a padded block carries a large diagonal shift in F', so
its levels sort above every real one and are never occupied.  All FP64.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from . import engine as E
from . import scf

E_CONV_DIIS, E_CONV, RMS_CONV, DIIS_CONV = 1e-11, 1e-13, 1e-10, 1e-10  # Constants.h:6-10
PAD_SHIFT = 1.0e4


class BatchSCF:
    """molecules: sequence of dicts with Z, xyz (bohr), basis, and optionally
    unrestricted (bool), alpha/beta electron counts (UHF).  concurrent_classes
    runs each batched build's classes on concurrent streams (on the 512-mix
    it was a wash: 20.2 vs 21.7 molecules/s)."""

    def __init__(self, molecules, unrestricted=False, alpha=0.75, init_guess=0.75, max_iter=300,
                 use_diis=True, schwarz_threshold=1e-12, device="cuda", concurrent_classes=False, graphs=False,
                 replay=8, eri_convention=E.ERI_REFERENCE, eigh_method=None):
        self.mols = list(molecules)
        self.uhf = unrestricted
        self.alpha, self.init_guess, self.max_iter, self.use_diis = alpha, init_guess, max_iter, use_diis
        # graphs: every SCF iteration after the DIIS history has filled is
        # captured once per working set as a CUDA graph (asynchronous batched
        # build on the device work queue, device DIIS solve, eigensolves,
        # density, energy, mixing and the convergence test, all on the
        # device) and replayed `replay` times between host checks of the
        # active count; converged molecules are frozen by the device mask
        self.graphs, self.replay = graphs, max(1, int(replay))
        self.graph_captures = 0
        self.dev = torch.device(device)
        self.eng = E.BatchEngine([(m["Z"], m["xyz"], m["basis"]) for m in self.mols],
                                 schwarz_threshold=schwarz_threshold, eri_convention=eri_convention)
        self.eng.set_streams(concurrent_classes)
        M = len(self.mols)
        self.M = M
        self.nbf = self.eng.nbf.astype(np.int64)
        self.nmax = int(self.nbf.max())
        n = self.nmax
        # one-electron matrices, S^-1/2, occupations, nuclear repulsion
        h = np.zeros((M, n, n))
        S = np.zeros((M, n, n))
        self.enuc = np.zeros(M)
        self.nocc = np.zeros((2, M), dtype=np.int64)
        for m, mol in enumerate(self.mols):
            k = int(self.nbf[m])
            Sm, hm = scf.one_electron(mol["Z"], mol["xyz"], mol["basis"])
            h[m, :k, :k], S[m, :k, :k] = hm, Sm
            self.enuc[m] = _nuclear_repulsion(mol["Z"], mol["xyz"])
            ne = int(sum(mol["Z"]))
            if unrestricted:
                na = mol.get("alpha_electrons") or ne - ne // 2
                nb = mol.get("beta_electrons") or ne // 2
                self.nocc[:, m] = (na, nb)
            else:
                self.nocc[:, m] = (max(1, ne // 2), 0)
        self.h = torch.from_numpy(h).to(self.dev)
        self.S = torch.from_numpy(S).to(self.dev)
        valid = torch.zeros(M, n, device=self.dev, dtype=torch.bool)
        for m in range(M):
            valid[m, : int(self.nbf[m])] = True
        self.valid = valid
        # V = S^-1/2 (HartreeFockAlgorithm.cpp:48-59); the padded block of S
        # is set to the identity for the decomposition, then V's is zeroed
        Spad = self.S + torch.diag_embed((~valid).double())
        w, U = torch.linalg.eigh(Spad)
        V = U @ torch.diag_embed(w.rsqrt()) @ U.transpose(1, 2)
        mask2 = valid[:, :, None] & valid[:, None, :]
        self.V = 0.5 * (V + V.transpose(1, 2)) * mask2
        self.mask2 = mask2
        self.shift = torch.diag_embed((~valid).double() * PAD_SHIFT)
        # eigensolver: 0 cuSOLVER batched Jacobi (default), 1 one dsyevd per
        # matrix (the single-molecule SCF's solver).  For the bench's 66 UHF
        # doublets (OH and planar CH3, STO-3G / 6-31G) both give the
        # single-molecule energies within 6.3e-12 Eh; method 0 takes 0.4 s of
        # eigensolves against 3.5 s
        self.eigh_method = 0 if eigh_method is None else int(eigh_method)
        self.seconds = {"fock": 0.0, "diis": 0.0, "eigh": 0.0, "total": 0.0}

    # ---- the working set: molecules still iterating, padded to their largest
    def _maps(self, W, n):
        """flat (engine layout) <-> padded [len(W), n, n] index maps and the
        eigensolver buckets of the working set W: molecules grouped by their
        exact nbf, so each batched solve runs at the molecule's own size with
        no padded level in it (a large padded level would set the solver's
        tolerance relative to itself and cost the real levels digits)."""
        rows, flat = [], []
        for r, m in enumerate(W):
            k = int(self.nbf[m])
            i, j = np.meshgrid(np.arange(k), np.arange(k), indexing="ij")
            rows.append(r * n * n + i.ravel() * n + j.ravel())
            flat.append(self.eng.offset[m] + i.ravel() * k + j.ravel())
        pad_idx = torch.from_numpy(np.concatenate(rows)).to(self.dev)
        flat_idx = torch.from_numpy(np.concatenate(flat)).to(self.dev)
        nb = self.nbf[W]
        buckets = [(int(b), np.nonzero(nb == b)[0]) for b in np.unique(nb)]
        return pad_idx, flat_idx, buckets

    def _guess_fock(self, h, S):
        if self.init_guess > 0:
            d = torch.diagonal(h, dim1=1, dim2=2)
            return self.init_guess * S * (d[:, :, None] + d[:, None, :]) * 0.5
        return h.clone()

    def _eigh(self, Ft, active_np, buckets):
        """Batched eigensolve of the active molecules, bucket by bucket
        (hfg_eigh_batched); levels of padded rows and of inactive molecules
        stay at PAD_SHIFT with unit vectors."""
        Mw, n = Ft.shape[0], Ft.shape[1]
        w = torch.full((Mw, n), PAD_SHIFT, dtype=torch.float64, device=self.dev)
        U = torch.eye(n, dtype=torch.float64, device=self.dev).expand(Mw, n, n).clone()
        for b, idx in buckets:
            sel = idx[active_np[idx] != 0]
            if len(sel) == 0:
                continue
            t = torch.from_numpy(sel).to(self.dev)
            wb, Ub = E.eigh_batched(Ft[t, :b, :b].contiguous(), method=self.eigh_method)
            w[t, :b] = wb
            U[t, :b, :b] = Ub
        return w, U

    def run(self):
        # captured loop: closed shells with the batched Jacobi solver (the
        # per-matrix dsyevd synchronises with the host inside cuSOLVER and
        # cannot be captured); UHF batches run the host-driven loop
        self.graphs_used = self.graphs and self.dev.type == "cuda" and self.eigh_method == 0 and not self.uhf
        if self.graphs_used:
            return self._run_graphs()
        return self._run_eager()

    def _run_eager(self, keep_state=False):
        """The host-driven loop.  keep_state: no working-set compaction, and
        the device state at the end (densities, DIIS history, previous
        energies, the active mask) is returned for the captured loop."""
        M, dev = self.M, self.dev
        nspin = 2 if self.uhf else 1
        # working set W (molecule ids) padded to n; it shrinks to the
        # molecules still iterating once half of it has converged, so the
        # per-step tensor work follows the active count
        W, n = np.arange(M), self.nmax
        h, S, V, shift = self.h, self.S, self.V, self.shift
        nocc = self.nocc
        enuc = torch.from_numpy(self.enuc).to(dev)
        pad_idx, flat_idx, buckets = self._maps(W, n)
        P = [torch.zeros(M, n, n, dtype=torch.float64, device=dev) for _ in range(nspin)]
        P_out = [torch.zeros(M, self.nmax, self.nmax, dtype=torch.float64, device=dev) for _ in range(nspin)]
        diisF = [[] for _ in range(nspin)]
        diisE = [[] for _ in range(nspin)]
        energy = torch.full((M,), float("inf"), dtype=torch.float64, device=dev)
        iters = torch.zeros(M, dtype=torch.int64, device=dev)
        converged = torch.zeros(M, dtype=torch.bool, device=dev)
        prev = torch.full((M,), float("inf"), dtype=torch.float64, device=dev)
        active = torch.ones(M, dtype=torch.bool, device=dev)
        flatG = [torch.zeros(self.eng.total, dtype=torch.float64, device=dev) for _ in range(nspin)]
        builds = 0
        # this thread's stream only: in a serving process other threads' jobs
        # keep the device busy and must not be waited for
        sync = torch.cuda.current_stream(self.dev).synchronize if self.dev.type == "cuda" else (lambda: None)

        def tick():
            sync()
            return time.perf_counter()

        def to_flat(X):
            out = torch.zeros(self.eng.total, dtype=torch.float64, device=dev)
            out[flat_idx] = X.reshape(-1)[pad_idx]
            return out

        def to_pad(flat):
            out = torch.zeros(len(W) * n * n, dtype=torch.float64, device=dev)
            out[pad_idx] = flat[flat_idx]
            return out.reshape(len(W), n, n)

        t_start = tick()
        for it in range(self.max_iter):
            act = active.clone()
            active_np = act.cpu().numpy().astype(np.uint8)
            Wt = torch.from_numpy(W).to(dev)
            if it == 0:
                F0 = self._guess_fock(h, S)
                F = [F0.clone() for _ in range(nspin)]
                if self.uhf:  # UnrestrictedHartreeFock.cpp:214-219: asymmetry on the alpha guess
                    F[0][:, 0, 1] += 0.1
                    F[0][:, 1, 0] = F[0][:, 0, 1]
            else:
                t0 = tick()
                mask = np.zeros(M, dtype=np.uint8)
                mask[W] = active_np
                flatP = [to_flat(p) for p in P]
                if self.uhf:
                    self.eng.fock_uhf(flatP[0], flatP[1], flatG[0], flatG[1], active=mask)
                else:
                    self.eng.fock_rhf(flatP[0], flatG[0], active=mask)
                builds += 1
                F = [h + to_pad(g) for g in flatG]
                self.seconds["fock"] += tick() - t0
            if not self.uhf:
                F = [0.5 * (f + f.transpose(1, 2)) for f in F]
            used = torch.zeros(len(W), dtype=torch.bool, device=dev)
            err_est = torch.zeros(len(W), dtype=torch.float64, device=dev)
            t0 = tick()
            if self.use_diis and it > 0:
                for s in range(nspin):
                    err = S @ P[s] @ F[s] - F[s] @ P[s] @ S
                    diisF[s].append(F[s].clone())
                    diisE[s].append(err)
                    if len(diisF[s]) > 6:
                        diisF[s].pop(0)
                        diisE[s].pop(0)
                    if len(diisF[s]) >= 5:
                        F[s], est = _diis_extrapolate(diisF[s], diisE[s])
                        err_est = err_est + est
                        used[:] = True
            t1 = tick()
            self.seconds["diis"] += t1 - t0
            Pn, eps = [], []
            for s in range(nspin):
                Ft = V @ F[s] @ V + shift
                w, Cp = self._eigh(Ft, active_np, buckets)
                self.seconds["eigh"] += tick() - t1
                t1 = tick()
                C = V @ Cp
                occ = (torch.arange(n, device=dev)[None, :] <
                       torch.from_numpy(nocc[s][W]).to(dev)[:, None]).double()
                factor = 1.0 if self.uhf else 2.0
                Co = C * occ[:, None, :]
                Pn.append(factor * Co @ Co.transpose(1, 2))
                eps.append((w * occ).sum(1))
            if self.uhf:
                e = 0.5 * (((Pn[0] + Pn[1]) * h).sum((1, 2)) + eps[0] + eps[1])
            else:
                e = 0.5 * (Pn[0] * h).sum((1, 2)) + eps[0]
            e = e + enuc[Wt]
            rms = torch.sqrt(sum(((pn - p) ** 2).sum((1, 2)) for pn, p in zip(Pn, P)))
            for s in range(nspin):
                mix = torch.where(used[:, None, None], Pn[s], self.alpha * Pn[s] + (1 - self.alpha) * P[s])
                P[s] = torch.where(act[:, None, None], mix, P[s])
            energy[Wt] = torch.where(act, e, energy[Wt])
            dE = (prev[Wt] - e).abs()
            econv = E_CONV_DIIS if self.use_diis else E_CONV
            conv = (dE <= econv) & (rms < RMS_CONV) & (err_est < DIIS_CONV)
            iters[Wt] = torch.where(act, iters[Wt] + 1, iters[Wt])
            prev[Wt] = torch.where(act, e, prev[Wt])
            converged[Wt] = converged[Wt] | (act & conv)
            active = act & ~conv
            n_active = int(active.sum())
            if n_active == 0:
                break
            if n_active <= len(W) // 2 and not keep_state:  # compact the working set
                for s in range(nspin):
                    P_out[s][Wt, :n, :n] = P[s]
                keep = active.cpu().numpy().astype(bool)
                kt = torch.from_numpy(np.nonzero(keep)[0]).to(dev)
                W = W[keep]
                n_new = int(self.nbf[W].max())
                sl = (slice(None), slice(0, n_new), slice(0, n_new))
                P = [p[kt][sl] for p in P]
                diisF = [[x[kt][sl] for x in lst] for lst in diisF]
                diisE = [[x[kt][sl] for x in lst] for lst in diisE]
                Wt_new = torch.from_numpy(W).to(dev)
                h, S, V, shift = (t[Wt_new][sl].contiguous() for t in (self.h, self.S, self.V, self.shift))
                active = active[kt]
                n = n_new
                pad_idx, flat_idx, buckets = self._maps(W, n)
        Wt = torch.from_numpy(W).to(dev)
        for s in range(nspin):
            P_out[s][Wt, :n, :n] = P[s]
        self.seconds["total"] = tick() - t_start
        self.iterations = iters.cpu().numpy()
        self.converged = converged.cpu().numpy()
        self.builds = builds
        self.energies = energy.cpu().numpy()
        self.densities = P_out
        if keep_state:
            # six history slots, oldest first; missing ones are zero
            # placeholders that the next append pushes out
            hist = ([[torch.zeros_like(P[0]) for _ in range(6 - len(diisF[s]))] + list(diisF[s]) for s in range(nspin)],
                    [[torch.zeros_like(P[0]) for _ in range(6 - len(diisE[s]))] + list(diisE[s]) for s in range(nspin)])
            return {"P": P, "hist": hist, "prev": prev, "active": active.cpu().numpy().astype(bool),
                    "iterations": it + 1}
        return self.energies

    def _run_graphs(self):
        """The captured loop: iterations 0-5 (the DIIS history fills) run in
        the host-driven loop, then one iteration per working set is captured
        and replayed; the working set shrinks to the molecules still
        iterating (and is captured again) once half of it has converged."""
        M, dev = self.M, self.dev
        nspin = 2 if self.uhf else 1
        t_start = time.perf_counter()
        keep_hist = 6  # DIIS.h:9
        econv = E_CONV_DIIS if self.use_diis else E_CONV
        enuc_all = torch.from_numpy(self.enuc).to(dev)
        nocc_all = [torch.from_numpy(self.nocc[s]).to(dev) for s in range(nspin)]
        P_out = [torch.zeros(M, self.nmax, self.nmax, dtype=torch.float64, device=dev) for _ in range(nspin)]

        eager = BatchSCF.__new__(BatchSCF)
        eager.__dict__.update(self.__dict__)
        eager.max_iter = min(self.max_iter, keep_hist)
        state = eager._run_eager(keep_state=True)
        energy = torch.from_numpy(eager.energies).to(dev)
        iters = torch.from_numpy(eager.iterations).to(dev)
        converged = torch.from_numpy(eager.converged).to(dev)
        self.seconds = dict(eager.seconds)
        builds = eager.builds
        P, hist, prev, it = state["P"], state["hist"], state["prev"], state["iterations"]
        for s in range(nspin):
            P_out[s].copy_(eager.densities[s])
        active = torch.from_numpy(state["active"]).to(dev)
        W = np.nonzero(state["active"])[0]

        def step(st, diis_on):
            """One SCF iteration of the working set, device only."""
            st.was_active.copy_(st.active)
            st.mask.zero_()
            st.mask[st.Wt] = st.active.to(torch.uint8)
            for s in range(nspin):
                st.flatP[s].zero_()
                st.flatP[s][st.flat_idx] = st.P[s].reshape(-1)[st.pad_idx]
            if self.uhf:
                self.eng.fock_uhf_async(st.flatP[0], st.flatP[1], st.flatG[0], st.flatG[1], st.mask)
            else:
                self.eng.fock_rhf_async(st.flatP[0], st.flatG[0], st.mask)
            Mw, n = len(st.W), st.n
            F = []
            for s in range(nspin):
                g = torch.zeros(Mw * n * n, dtype=torch.float64, device=dev)
                g[st.pad_idx] = st.flatG[s][st.flat_idx]
                f = st.h + g.reshape(Mw, n, n)
                if not self.uhf:
                    f = 0.5 * (f + f.transpose(1, 2))
                F.append(f)
            err_est = torch.zeros(Mw, dtype=torch.float64, device=dev)
            if diis_on:
                for s in range(nspin):
                    err = st.S @ st.P[s] @ F[s] - F[s] @ st.P[s] @ st.S
                    # the history, oldest first: drop the oldest, append this one
                    st.hist_F[s][:-1] = st.hist_F[s][1:].clone()
                    st.hist_E[s][:-1] = st.hist_E[s][1:].clone()
                    st.hist_F[s][-1] = F[s]
                    st.hist_E[s][-1] = err
                    Ee = st.hist_E[s].transpose(0, 1)  # [Mw, keep, n, n]
                    B = torch.einsum("aikl,ajkl->aij", Ee, Ee)
                    m = keep_hist
                    Bb = torch.zeros(Mw, m + 1, m + 1, dtype=torch.float64, device=dev)
                    Bb[:, :m, :m] = B
                    Bb[:, m, :m] = 1
                    Bb[:, :m, m] = 1
                    c = E.pulay_solve_device(Bb)[:, :m]
                    F[s] = torch.einsum("ai,iakl->akl", c, st.hist_F[s])
                    err_est = err_est + torch.sqrt(torch.diagonal(B, dim1=1, dim2=2)[:, -2:].sum(1))
            Pn, eps = [], []
            for s in range(nspin):
                st.Ft.copy_(st.V @ F[s] @ st.V + st.shift)
                for b, idx in st.bucket_idx:
                    wb, Ub = E.eigh_batched(st.Ft[idx, :b, :b].contiguous(), method=self.eigh_method)
                    st.w[idx, :b] = wb
                    st.U[idx, :b, :b] = Ub
                C = st.V @ st.U
                factor = 1.0 if self.uhf else 2.0
                Co = C * st.occ[s][:, None, :]
                Pn.append(factor * Co @ Co.transpose(1, 2))
                eps.append((st.w * st.occ[s]).sum(1))
            if self.uhf:
                e = 0.5 * (((Pn[0] + Pn[1]) * st.h).sum((1, 2)) + eps[0] + eps[1])
            else:
                e = 0.5 * (Pn[0] * st.h).sum((1, 2)) + eps[0]
            e = e + st.enuc
            rms = torch.sqrt(sum(((pn - p) ** 2).sum((1, 2)) for pn, p in zip(Pn, st.P)))
            act = st.was_active
            for s in range(nspin):
                mix = Pn[s] if diis_on else self.alpha * Pn[s] + (1 - self.alpha) * st.P[s]
                st.P[s].copy_(torch.where(act[:, None, None], mix, st.P[s]))
            st.e.copy_(torch.where(act, e, st.e))
            dE = (st.prev - e).abs()
            st.conv.copy_(act & (dE <= econv) & (rms < RMS_CONV) & (err_est < DIIS_CONV))
            st.prev.copy_(torch.where(act, e, st.prev))
            st.active.copy_(act & ~st.conv)
            st.converged.copy_(st.converged | st.conv)
            st.iters.copy_(st.iters + act.long())

        while len(W) and it < self.max_iter:
            n = int(self.nbf[W].max())
            sl = (slice(None), slice(0, n), slice(0, n))
            st = _GraphState()
            st.W, st.n = W, n
            st.Wt = torch.from_numpy(W).to(dev)
            Mw = len(W)
            st.h, st.S, st.V, st.shift = (t[st.Wt][sl].contiguous() for t in (self.h, self.S, self.V, self.shift))
            st.pad_idx, st.flat_idx, buckets = self._maps(W, n)
            st.bucket_idx = [(b, torch.from_numpy(idx).to(dev)) for b, idx in buckets]
            st.P = [p[st.Wt][sl].contiguous() for p in P]
            st.hist_F = [torch.stack([x[st.Wt][sl] for x in hist[0][s]], 0).contiguous() for s in range(nspin)]
            st.hist_E = [torch.stack([x[st.Wt][sl] for x in hist[1][s]], 0).contiguous() for s in range(nspin)]
            st.prev = prev[st.Wt].contiguous()
            st.active = active[st.Wt].contiguous()
            st.enuc = enuc_all[st.Wt].contiguous()
            st.occ = [(torch.arange(n, device=dev)[None, :] < nocc_all[s][st.Wt][:, None]).double()
                      for s in range(nspin)]
            st.flatP = [torch.zeros(self.eng.total, dtype=torch.float64, device=dev) for _ in range(nspin)]
            st.flatG = [torch.zeros(self.eng.total, dtype=torch.float64, device=dev) for _ in range(nspin)]
            st.mask = torch.zeros(M, dtype=torch.uint8, device=dev)
            st.e = energy[st.Wt].contiguous()
            st.conv = torch.zeros(Mw, dtype=torch.bool, device=dev)
            st.was_active = torch.zeros(Mw, dtype=torch.bool, device=dev)
            st.converged = torch.zeros(Mw, dtype=torch.bool, device=dev)
            st.iters = torch.zeros(Mw, dtype=torch.int64, device=dev)
            st.Ft = torch.zeros(Mw, n, n, dtype=torch.float64, device=dev)
            st.w = torch.full((Mw, n), PAD_SHIFT, dtype=torch.float64, device=dev)
            st.U = torch.eye(n, dtype=torch.float64, device=dev).expand(Mw, n, n).clone()
            step(st, self.use_diis)  # eager warm-up of this shape (allocations, workspaces)
            it += 1
            builds += 1
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(side):
                with torch.cuda.graph(g):
                    step(st, self.use_diis)
            torch.cuda.current_stream().wait_stream(side)
            self.graph_captures += 1
            while it < self.max_iter:
                k = min(self.replay, self.max_iter - it)
                for _ in range(k):
                    g.replay()
                it += k
                builds += k
                n_act = int(st.active.sum())
                if n_act == 0 or n_act <= Mw // 2:
                    break
            # results of the working set, and the state of the molecules still
            # iterating for the next (smaller) one
            energy[st.Wt] = st.e
            iters[st.Wt] += st.iters
            converged[st.Wt] |= st.converged
            for s in range(nspin):
                P_out[s][st.Wt, :n, :n] = st.P[s]
            act_now = st.active.cpu().numpy().astype(bool)
            P = [torch.zeros(M, self.nmax, self.nmax, dtype=torch.float64, device=dev) for _ in range(nspin)]
            hist = ([[torch.zeros(M, self.nmax, self.nmax, dtype=torch.float64, device=dev)
                      for _ in range(keep_hist)] for _ in range(nspin)],
                    [[torch.zeros(M, self.nmax, self.nmax, dtype=torch.float64, device=dev)
                      for _ in range(keep_hist)] for _ in range(nspin)])
            for s in range(nspin):
                P[s][st.Wt, :n, :n] = st.P[s]
                for j in range(keep_hist):
                    hist[0][s][j][st.Wt, :n, :n] = st.hist_F[s][j]
                    hist[1][s][j][st.Wt, :n, :n] = st.hist_E[s][j]
            prev = torch.full((M,), float("inf"), dtype=torch.float64, device=dev)
            prev[st.Wt] = st.prev
            active = torch.zeros(M, dtype=torch.bool, device=dev)
            active[st.Wt] = st.active
            W = W[act_now]
            del g
        torch.cuda.synchronize()
        self.seconds["total"] = time.perf_counter() - t_start
        self.iterations = iters.cpu().numpy()
        self.converged = converged.cpu().numpy()
        self.builds = builds
        self.energies = energy.cpu().numpy()
        self.densities = P_out
        return self.energies


class _GraphState:
    """Device state of one working set for the captured iteration: every
    tensor a replay reads or writes keeps its storage for the life of the
    graph."""


def _diis_extrapolate(Fs, Es):
    """Pulay extrapolation per molecule (DIIS.h:34-96): B_ij = <e_i, e_j>,
    bordered by ones; returns sum_i c_i F_i and sqrt(|e_m|^2 + |e_m-1|^2)."""
    m = len(Fs)
    Ee = torch.stack(Es, 1)  # [M, m, n, n]
    B = torch.einsum("aikl,ajkl->aij", Ee, Ee)
    M = B.shape[0]
    Bb = torch.zeros(M, m + 1, m + 1, dtype=B.dtype, device=B.device)
    Bb[:, :m, :m] = B
    Bb[:, m, :m] = 1
    Bb[:, :m, m] = 1
    # the (m+1)^2 systems are tiny and turn rank-deficient near convergence:
    # solved on the host by the SCF's own column-pivoted QR (DIIS.h:72),
    # which also decides the reference's extrapolation there
    c = torch.from_numpy(scf.pulay_solve(Bb.cpu().numpy())[:, :m]).to(B.device)
    F = torch.einsum("ai,aikl->akl", c, torch.stack(Fs, 1))
    est = torch.sqrt(torch.diagonal(B, dim1=1, dim2=2)[:, -2:].sum(1))
    return F, est


def _nuclear_repulsion(Z, xyz):
    xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    e = 0.0
    for a in range(len(Z)):
        for b in range(a):
            e += Z[a] * Z[b] / np.linalg.norm(xyz[a] - xyz[b])
    return e
