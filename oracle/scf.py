"""CPU oracle of the SCF set-up and potential update (test infrastructure
only: tests/, the smoke check and the bench's CPU leg use it; the library
never does).

A restatement in numpy of the reference routines, each function citing the
one it follows:

  lattice_points     getNumCells / makeLattice / cellBorderCheck / mergeSort
                     (lattice.f90:469-782, sortSubs.f90:18-200)
  electrostatics     neutralAndNuclearQPot, residualQ (elecStat.f90:59-1042)
  mesh               makeSampleVectors, getECMeshParameters,
                     makeECMeshAndOverlap (exchCorr.f90:63-980)
  core_rho           makeCoreRho (coreCharge.f90:27-578)
  make_scf_pot       makeSCFPot for spin 1, rel 0, LDA (potentialUpdate.F90:53-1866)

It is checked against fixtures made by executing the reference's own
statements (tests/golden/make_scf_golden.py); the library is checked
against both.  Sizes: seconds for cells of a few atoms.
"""
import math

import numpy as np

PI = 3.141592653589793
SMALL = 1.0e-8


def f32(x):
    return float(np.float32(x))


# ---------------------------------------------------------------- lattice

def ref_merge_order(keys):
    """mergeSort's permutation (sortSubs.f90:18-200): bottom-up merges of
    neighbouring runs; a head of the first run goes first only when strictly
    smaller than the second run's head."""
    order = list(range(len(keys)))
    runs = [[i] for i in order]
    while len(runs) > 1:
        nxt = []
        for r in range(0, len(runs) - 1, 2):
            a, b = runs[r], runs[r + 1]
            i = j = 0
            m = []
            while i < len(a) and j < len(b):
                if keys[a[i]] < keys[b[j]]:
                    m.append(a[i])
                    i += 1
                else:
                    m.append(b[j])
                    j += 1
            m += a[i:] + b[j:]
            nxt.append(m)
        if len(runs) % 2:
            nxt.append(runs[-1])
        runs = nxt
    return runs[0] if runs else []


def lattice_points(vectors, lim):
    """vectors: rows a, b, c (xyz).  Returns (dims [n, 3], sizes [n])."""
    v = np.asarray(vectors, float)
    reps = [2 * math.ceil(math.sqrt(lim) / math.sqrt(float(v[i] @ v[i]))) + 1 for i in range(3)]
    shift = v.sum(axis=0)
    pts, sizes = [], []
    for i in range(1, reps[0] + 1):
        for j in range(1, reps[1] + 1):
            for k in range(1, reps[2] + 1):
                rep = (i - (1 + reps[0]) // 2, j - (1 + reps[1]) // 2, k - (1 + reps[2]) // 2)
                t = [0.0, 0.0, 0.0]
                for l in range(3):
                    for m in range(3):
                        t[m] = t[m] + v[l, m] * rep[l]
                s = t[0] * t[0] + t[1] * t[1] + t[2] * t[2]
                if s > lim:
                    cur = list(t)
                    ok = False
                    for ax, sg in ((0, 1), (1, 1), (0, -1), (2, 1), (0, 1), (1, -1), (0, -1)):
                        cur[ax] += sg * shift[ax]
                        if cur[0] ** 2 + cur[1] ** 2 + cur[2] ** 2 < lim:
                            ok = True
                            break
                    if not ok:
                        continue
                pts.append(t)
                sizes.append(s)
    o = ref_merge_order(sizes)
    return np.array(pts)[o], np.array(sizes)[o]


def recip_vectors(rv):
    rv = np.asarray(rv, float)
    rec = np.zeros((3, 3))
    vol = 0.0
    for i in range(3):
        vol = 0.0
        i1, i2 = (i + 1) % 3, (i + 2) % 3
        for j in range(3):
            j1, j2 = (j + 1) % 3, (j + 2) % 3
            rec[i, j] = rv[i1, j1] * rv[i2, j2] - rv[i1, j2] * rv[i2, j1]
            vol = vol + rec[i, j] * rv[i, j]
        rec[i] = 2.0 * PI * rec[i] / vol
    return rec, abs(vol)


def nearest(rv, v):
    rv = np.asarray(rv, float)
    f = np.linalg.solve(rv.T, v)
    base = np.trunc(np.abs(f) + 0.5) * np.sign(f)
    best, bd = None, None
    for d in np.ndindex(3, 3, 3):
        L = (base + np.array(d) - 1) @ rv
        x = float(((v - L) ** 2).sum())
        if bd is None or x < bd * (1 - 1e-12):
            best, bd = L, x
    return best


def ref_erf(x):
    """error_fn (mathSubs.f90:22-140) on an array."""
    x = np.asarray(x, float)
    ax = np.abs(x)
    out = np.where(ax > 6.0, np.sign(x), 0.0)
    x2 = ax * ax
    m = ax <= 0.46875
    a = ax * (242.6679552305318 + x2 * (21.97926161829415 + x2 * (6.996383488619136 +
                                                                  x2 * -0.03560984370181539)))
    a = a / (215.0588758698612 + x2 * (91.16490540451490 + x2 * (15.08279763040779 + x2)))
    out = np.where(m, np.where(x < 0, -a, a), out)
    m2 = (ax > 0.46875) & (ax <= 4.0)
    b = np.exp(-x2) * (22.898992851659 + ax * (26.094746956075 + ax * (
        14.571898596926 + ax * (4.2677201070898 + ax * (0.56437160686381 +
                                                         ax * -0.0000060858151959688)))))
    b = b / (22.898985749891 + ax * (51.933570687552 + ax * (50.273202863803 + ax * (
        26.288795758761 + ax * (7.5688482293618 + ax)))))
    out = np.where(m2, np.copysign(1.0 - b, x), out)
    m3 = (ax > 4.0) & (ax <= 6.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / x2
        c = inv * (-0.0121308276389978 + inv * (-0.119903955268146 + inv * (
            -0.243911029488626 + inv * -0.0324319519277746)))
        c = c / (0.043002664345277 + inv * (0.489552441961437 + inv * (1.43771227937118 + inv)))
        c = np.exp(-x2) * (0.564189583547756 + c) / ax
    return np.where(m3, np.copysign(1.0 - c, x), out)


class ScfOracle:
    """The set-up of one system; pot_types/sites as the system holds them."""

    def __init__(self, system, num_sample_vectors=100, weights=(0.5, 0.5),
                 r_sample=(0.1, 3.5, 0.8)):
        s = system
        self.s = s
        self.rv = np.asarray(s.real_vectors, float)
        self.rec, self.volume = recip_vectors(self.rv)
        self.Tb = -math.log(s.basis_fn_convg)
        self.Te = -math.log(s.electro_convg)
        self.alphas = [np.asarray(p.alphas, float) for p in s.pot_types]
        self.off = np.cumsum([0] + [len(a) for a in self.alphas])[:-1]
        self.P = int(sum(len(a) for a in self.alphas))
        self.ptype = np.asarray(s.pot_site_type) - 1
        self.pos = np.asarray(s.pot_site_pos, float)
        self.mult = np.array([(self.ptype == t).sum() for t in range(len(self.alphas))])
        min_atom = min(100.0, *[t.alphas[0] for t in s.atom_types])
        self.min_pot = min(10000.0, *[a[0] for a in self.alphas])
        lim = self.Tb * max(2.0 / min_atom, 1.0 / self.min_pot + 0.5 / min_atom)
        maxsq = max(float(v @ v) for v in self.rv)
        lim = lim + 0.75 * maxsq + math.sqrt(3.0 * maxsq * lim)
        lim = max(lim, 2.0 * self.Tb / min_atom)
        self.cells, self.csize = lattice_points(self.rv, lim)
        self.rcells, self.rcsize = lattice_points(self.rec, 4.0 * self.Te * self.min_pot)
        self.intg = np.concatenate([m * PI ** 1.5 / a ** 1.5
                                    for m, a in zip(self.mult, self.alphas)])
        self.electrostatics()
        self.core_rho()
        self.mesh(num_sample_vectors, weights, r_sample)

    # ------------------------------------------------------ electrostatics
    def electrostatics(self):
        """neutralAndNuclearQPot (elecStat.f90:249-520) and residualQ
        (elecStat.f90:794-1005)."""
        P, T = self.P, self.Te
        nl = np.zeros((P, P))
        loc = np.zeros((P, P))
        ol = np.zeros((P, P))
        nuc = np.zeros(P)
        lnuc = np.zeros(P)
        ntyp = len(self.alphas)
        res = np.zeros((ntyp, P))
        # residualQ's tables, recomputed only when the element changes
        tabs = {}
        last_el, cur = 0, None
        for t, p in enumerate(self.s.pot_types):
            if p.element != last_el:
                a = self.alphas[t]
                mu = a * self.min_pot / (a + self.min_pot)
                G2 = self.rcsize[1:]
                cur = (np.sqrt(mu), np.exp(-np.outer(G2, 0.25 / mu)) / G2[:, None])
            last_el = p.element
            tabs[t] = cur
        for i in range(len(self.pos)):
            t1 = self.ptype[i]
            a1 = self.alphas[t1]
            n1, o1 = len(a1), self.off[t1]
            for j in range(len(self.pos)):
                t2 = self.ptype[j]
                a2 = self.alphas[t2]
                n2, o2 = len(a2), self.off[t2]
                sep = self.pos[i] - self.pos[j]
                ms = sep - nearest(self.rv, sep)
                d = ms[None, :] - self.cells
                r2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
                r = np.sqrt(r2)
                X1, X2 = np.meshgrid(a1, a2, indexing="ij")
                rpa = X1 * X2 / (X1 + X2)
                nq = PI ** 3 / (X1 * np.sqrt(X1) * X2 * np.sqrt(X2))
                oc = (PI / (X1 + X2)) ** 1.5
                nmin = min(n1, n2)
                diag = a1[:nmin] * a2[:nmin] / (a1[:nmin] + a2[:nmin])
                # first failing diagonal per cell (nmin - 1 if none)
                if nmin >= 2:
                    fail = diag[None, :nmin - 1] * r2[:, None] > T
                    first = np.where(fail.any(axis=1), fail.argmax(axis=1), nmin - 1)
                else:
                    first = np.full(len(r2), 10 ** 6)
                mn = np.minimum.outer(np.arange(n1), np.arange(n2))
                for c in range(len(r2)):
                    inc = mn < first[c] if first[c] < nmin - 1 else np.ones_like(mn, bool)
                    if not inc.any():
                        continue
                    if abs(r2[c]) >= SMALL:
                        v = nq / r[c] * (-ref_erf(np.sqrt(X1) * r[c]) + ref_erf(np.sqrt(rpa) * r[c]))
                        nl[o2:o2 + n2, o1:o1 + n1] += np.where(inc, v, 0.0).T
                    else:
                        v = nq * (2.0 / math.sqrt(PI)) * np.sqrt(rpa)
                        loc[o2:o2 + n2, o1:o1 + n1] += np.where(inc, v, 0.0).T
                    ol[o2:o2 + n2, o1:o1 + n1] += np.where(inc, oc * np.exp(-rpa * r2[c]), 0.0).T
                nuca, z2 = self.s.pot_types[t2].nuc_alpha, self.s.pot_types[t2].nuc_charge
                nf = a1 + nuca
                for c in range(len(r2)):
                    for m in range(n1):
                        scr = r2[c] * a1[m] * nuca / nf[m]
                        if not scr < T:
                            break
                        if abs(scr) >= SMALL:
                            co = a1[m] * r[c] / math.sqrt(nf[m])
                            nuc[o1 + m] -= (z2 * PI ** 1.5 * math.exp(-scr) * float(ref_erf(co))
                                            / co / nf[m])
                        else:
                            nuc[o1 + m] -= z2 * math.exp(-scr) * (2 * PI) / nf[m]
                if float(sep @ sep) < SMALL:
                    lnuc[o1:o1 + n1] -= 2 * PI * self.s.pot_types[t1].nuc_charge / a1
                # residualQ
                mra, rce = tabs[t1]
                a21 = a2[0]
                f1 = PI ** 1.5 / (a1 * np.sqrt(a1))
                f2 = PI ** 1.5 / (a21 * math.sqrt(a21))
                af = f1 * f2
                rps = np.sqrt(a1 * a21 / (a1 + a21))
                self_f = 2.0 / math.sqrt(PI) * af * (rps - mra[:n1])
                vf = 4.0 * PI * af / self.volume
                ph = np.cos(self.rcells[1:] @ sep)
                sqT = math.sqrt(T)
                for k in range(n1):
                    acc = 0.0
                    for c in range(len(r2)):
                        if r2[c] < SMALL:
                            acc += self_f[k]
                        else:
                            if mra[k] * r[c] > sqT and rps[k] * r[c] > sqT:
                                break
                            acc += af[k] * (-float(ref_erf(mra[k] * r[c]))
                                            + float(ref_erf(rps[k] * r[c]))) / r[c]
                    acc += vf[k] * (float(rce[:, k] @ ph) - 0.25 / self.min_pot)
                    res[t2, o1 + k] += acc
        self.pot_ol, self.nl_neut, self.l_neut = ol, nl, loc
        self.nl_nuc, self.l_nuc, self.nl_res = nuc, lnuc, res

    # ------------------------------------------------------------ core rho
    def core_rho(self):
        """makeCoreRho (coreCharge.f90:27-578)."""
        out = np.zeros(self.P)
        fac = np.array([math.sqrt(PI) * n / d * (2 * k + 1) * 2.0 * 2.0
                        for k, (n, d) in enumerate(((1, 4), (3, 8), (15, 16), (105, 32)))])
        seen = set()
        for i in range(len(self.pos)):
            t = int(self.ptype[i])
            if t in seen:
                continue
            seen.add(t)
            if t >= len(self.s.atom_types):
                continue
            at = self.s.atom_types[t]
            if not at.core_l:
                continue
            pa = self.alphas[t]
            np_ = len(pa)
            aa = np.asarray(at.alphas, float)
            noa = at.num_orb_alphas
            ov = np.zeros((np_, 2))
            for j in range(np_):
                ov[j, 1] = PI ** 1.5 / pa[j] ** 1.5
                o1 = 0.0
                for l_, cf in zip(at.core_l, at.core_coeffs):
                    n = noa[l_]
                    for a in range(n):
                        for b in range(a, n):
                            rg = 1.0 / (pa[j] + aa[a] + aa[b])
                            o1 += fac[l_] * math.sqrt(rg) * rg ** (l_ + 1) * cf[a] * cf[b]
                        rg = 1.0 / (pa[j] + aa[a] + aa[a])
                        o1 -= fac[l_] * math.sqrt(rg) * rg ** (l_ + 1) * cf[a] * cf[a] * 0.5
                ov[j, 0] = o1
            S = PI ** 1.5 / (pa[:, None] + pa[None, :]) ** 1.5
            x = dposvx(S, ov)
            ints = ov[:, 1]
            ne = 2.0 * at.num_core_states
            delta = (ne - float(x[:, 0] @ ints)) / float(x[:, 1] @ ints)
            out[self.off[t]:self.off[t] + np_] = x[:, 0] + delta * x[:, 1]
        self.core = out

    # ----------------------------------------------------------------- mesh
    def mesh(self, nv, wt, rs):
        """makeSampleVectors, getECMeshParameters and makeECMeshAndOverlap
        (exchCorr.f90:63-980)."""
        h = np.array([-1.0] + [-1.0 + 2.0 * k / (nv - 1.0) for k in range(1, nv - 1)] + [1.0])
        th = np.arccos(h)
        ph = np.zeros(nv)
        for k in range(1, nv - 1):
            ph[k] = ph[k - 1] + 3.6 / math.sqrt(nv) * 1.0 / math.sqrt(1.0 - h[k] * h[k])
            while ph[k] > 2.0 * PI:
                ph[k] -= 2.0 * PI
        vec = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], axis=1)
        cov = np.array([p.covalent_radius for p in self.s.pot_types])
        ns = len(self.pos)
        nreps = min(64, len(self.csize))
        live = [cov[self.ptype[i]] >= SMALL for i in range(ns)]
        lsep = np.zeros((ns, 3))
        lst = np.zeros((ns, nreps, 3))
        for i in range(ns):
            if live[i]:
                lsep[i] = self.pos[i] - nearest(self.rv, self.pos[i])
                lst[i] = lsep[i] + self.cells[:nreps]
        maxr = math.sqrt(rs[1] / self.min_pot)
        pts, ws, counts = [], [], []
        space = rs[2]
        wf = (1.0 - space) / math.sqrt(space)
        for i in range(ns):
            if not live[i]:
                counts.append(0)
                continue
            ci = cov[self.ptype[i]]
            a = self.alphas[self.ptype[i]]
            half, minr = ci / 2.0, math.sqrt(rs[0] / a[-1])
            n0 = len(ws)
            for j in range(nv):
                cur = maxr
                for k in range(ns):
                    if not live[k]:
                        continue
                    f = ci / (ci + cov[self.ptype[k]])
                    sep = f * (lst[k] - lst[i, 0])
                    dot = sep @ vec[j]
                    for l in range(nreps):
                        if dot[l] <= SMALL:
                            continue
                        cur = min(float(sep[l] @ sep[l]) / dot[l], cur)
                r, wi, endf = cur, 1, 0.5
                while True:
                    pts.append(r * vec[j] + lsep[i])
                    ws.append(wt[wi] * wf * endf * (r * r * r))
                    endf = 1.0
                    if r < half or r < minr:
                        wi = 0
                    if wt[wi] < SMALL:
                        break
                    if r < minr:
                        r = r * math.sqrt(space)
                        pts.append(0.75 * r * vec[j] + lsep[i])
                        ws.append(wt[0] * (r * r * r) / 3.0)
                        break
                    r = r * space
            counts.append(len(ws) - n0)
        pts = np.array(pts)
        op = np.zeros((len(pts), self.P))
        T = self.Te
        for l in range(ns):
            t = self.ptype[l]
            a = self.alphas[t]
            neg = T / a[0]
            for p, x in enumerate(pts):
                v = x - self.pos[l]
                off = v - nearest(self.rv, v)
                m2 = float(off @ off)
                plus = neg + m2 + 2.0 * math.sqrt(neg * m2)
                ncell = int(np.searchsorted(self.csize, plus, side="right"))
                d = off[None, :] - self.cells[:ncell]
                r2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
                r2 = r2[r2 <= neg]
                e = np.outer(r2, a)
                keep = np.cumprod(e <= T, axis=1).astype(bool)
                op[p, self.off[t]:self.off[t] + len(a)] += np.where(keep, np.exp(-e), 0.0).sum(axis=0)
        self.points, self.weights, self.site_points = pts, np.array(ws), np.array(counts)
        self.op = op
        self.xc_ol = np.triu((op * self.weights[:, None]).T @ op)

    # ------------------------------------------------------------- update
    def reset(self):
        self.hist = None
        self.iteration = 1

    def make_scf_pot(self, pot_rho, nuc_trace, kin_trace, coeffs, num_electrons, xc=100,
                     feedback=2, relax=0.2, convg=1e-4):
        """makeSCFPot (potentialUpdate.F90:53-1866), spin 1, rel 0.  Returns
        (next coefficients, {totalEnergy, kineticEnergy, elecStatEnergy,
        exchCorrEnergy, electronDiff, testableDelta, converged})."""
        if not hasattr(self, "hist"):
            self.reset()
        P = self.P
        S = self.pot_ol
        g = dposvx(S, np.stack([pot_rho, self.intg], axis=1))
        g1, g2 = g[:, 0], g[:, 1]
        ediff = num_electrons - float(self.intg @ g1)
        g2 = g1 + g2 * ediff / float(self.intg @ g2)
        g3 = self.core.copy()
        g1 = g2 + g3
        g4 = g1.copy()
        g5, g6, g7 = np.zeros(P), np.zeros(P), np.zeros(P)
        for t, a in enumerate(self.alphas):
            b, e = self.off[t], self.off[t] + len(a) - 1
            zc = self.s.pot_types[t].nuc_charge * self.mult[t]
            sm = float(self.intg[b:e + 1] @ g1[b:e + 1])
            g5[b] = (sm - zc) / self.intg[b]
            g4[b] = g1[b] - g5[b]
            g6[t] = g5[b]
            g7[e] = -zc / self.intg[e]
        es1 = self.nl_neut.T @ g4
        es2 = self.l_neut.T @ (g2 - g5)
        es3 = self.l_neut.T @ g3
        es4, es5 = self.nl_nuc, self.l_nuc
        es6 = self.nl_res.T @ g6[:len(self.alphas)]
        e_es = float(np.sum(0.5 * (g1 + g7) * (es1 + es6) + 0.5 * g2 * (es2 + es3 + es5)
                            + 0.5 * (g2 - g5) * (es3 + es5)))
        e_es = e_es - float(g2 @ es4) + nuc_trace
        pot = dposvx(S, np.stack([es1 + es2 + es3 - es4 + es5, es6], axis=1))
        tot = np.maximum(self.op @ g1, 0.0)
        core = np.maximum(self.op @ g3, 0.0)
        v1, v2 = lda(tot, xc)
        _, v3 = lda(core, xc)
        xcp = (self.op * self.weights[:, None]).T @ np.stack([v1, v2, v3], axis=1)
        xcp = dposvx(self.xc_ol, xcp)
        e_xc = float((S @ xcp[:, 1]) @ g1 - (S @ xcp[:, 2]) @ g3)
        total = kin_trace + e_es + e_xc
        res = {"totalEnergy": total, "kineticEnergy": kin_trace, "elecStatEnergy": e_es,
               "exchCorrEnergy": e_xc, "electronDiff": ediff}
        if total > 0.0:
            raise ValueError("Total energy is positive!")
        x0 = np.asarray(coeffs, float)
        y0 = pot[:, 0] + pot[:, 1] + xcp[:, 0]
        if self.hist is None:
            self.hist = [x0.copy(), x0.copy(), y0.copy(), y0.copy()]
        xl1, xl2, yl1, yl2 = self.hist
        out = y0 - x0
        delta = 0.0
        o = 0
        for n in self.site_points:
            if n:
                d = self.op[o:o + n] @ out
                w = self.weights[o:o + n]
                delta = max(math.sqrt(float(np.sum(w * d * d)) / float(np.sum(w))), delta)
            o += n
        th1 = th2 = 0.0
        if feedback and self.iteration > 1:
            r0, r1, r2 = y0 - x0, yl1 - xl1, yl2 - xl2
            d1, d2 = r0 - r1, r0 - r2
            s11, t1 = float(d1 @ S @ d1), float(d1 @ S @ r0)
            s12, s22, t2 = float(d2 @ S @ d1), float(d2 @ S @ d2), float(d2 @ S @ r0)
            th1 = t1 / s11
            if feedback != 1 and self.iteration > 2:
                det = s11 * s22 - s12 * s12
                if det / (s11 * s22) >= 0.01:
                    th1 = (s22 * t1 - s12 * t2) / det
                    th2 = (-s12 * t1 + s11 * t2) / det
        nxt = (1.0 - relax) * ((1.0 - th1 - th2) * x0 + th1 * xl1 + th2 * xl2) + \
            relax * ((1.0 - th1 - th2) * y0 + th1 * yl1 + th2 * yl2)
        self.hist = [x0.copy(), xl1, y0.copy(), yl1]
        conv = int(delta < convg)
        if not conv:
            self.iteration += 1
        res.update(testableDelta=delta, converged=conv, currIteration=self.iteration)
        return nxt, res


def dposvx(A, B):
    """solveDPOSVX (interfaces.F90:236-293): LAPACK dposvx('E', 'U')."""
    from scipy.linalg import lapack
    B = np.asarray(B, float)
    b = B.reshape(B.shape[0], -1)
    x = lapack.dposvx(np.triu(np.asarray(A, float)), b, fact="E", lower=0)
    if x[9] != 0:
        raise ValueError(f"dposvx failed, info {x[9]}")
    return x[5].reshape(B.shape)


def lda(rho, xc):
    """The local-density functionals of makeSCFPot (potentialUpdate.F90:
    2835-3123): (potential, energy density) per point; the single-precision
    literals as gfortran stores them."""
    rho = np.asarray(rho, float)
    if xc == 100:
        r13 = rho ** 0.3333333333333333333
        f = 1.0 + 12.57 * r13
        return (-r13 * (0.984 + (0.943656 + 8.8963 * r13) / f ** 2),
                -0.738 * r13 * (1.0 + 0.959 / f))
    third = f32(0.33333333)
    with np.errstate(divide="ignore", invalid="ignore"):
        alpha = (4.0 / (9.0 * PI)) ** third
        rs = np.where(rho < SMALL, 1.0, (3.0 / (4.0 * PI * np.maximum(rho, SMALL))) ** third)
        if xc == 101:
            ex = -3.0 / (2.0 * PI * alpha) / rs
            g, b1, b2 = f32(-0.1423), f32(1.0529), f32(0.3334)
            sq = np.sqrt(rs)
            ec = g / (1 + b1 * sq + b2 * rs)
            hi_e = ex + ec
            hi_p = f32(4.0 / 3.0) * ex + ec * ec / g * (1 + f32(7.0 / 6.0) * b1 * sq
                                                        + f32(4.0 / 3.0) * b2 * rs)
            af, bf, cf, df = f32(0.0311), f32(-0.0480), f32(0.0020), f32(-0.0116)
            ln = np.log(rs)
            lo_e = ex + af * ln + bf + cf * rs * ln + df * rs
            lo_p = (f32(4.0 / 3.0) * ex + af * ln + (bf - f32(1.0 / 3.0) * af)
                    + f32(2.0 / 3.0) * cf * rs * ln + f32(1.0 / 3.0) * (2 * df - cf) * rs)
            pot = np.where(rs >= 1.0, hi_p, lo_p) * f32(0.5)
            en = np.where(rs >= 1.0, hi_e, lo_e) * f32(0.5)
        else:
            x = rs / 21.0
            lg = np.log(1.0 + 1.0 / x)
            pot = (-2.0 / (PI * alpha * rs) - 0.045 * lg) * f32(0.5)
            en = (-0.75 * 2.0 / (PI * alpha * rs)
                  - 0.045 * ((1 + x ** 3.0) * lg + x / 2.0 - x ** 2.0 - third)) * f32(0.5)
    small = rho < SMALL
    return np.where(small, 0.0, pot), np.where(small, 0.0, en)
