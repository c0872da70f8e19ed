"""Generator of the per-class contracted-ERI device functions.

For every shell-quartet class of the direct-SCF Fock build this emits one
straight-line CUDA device function that evaluates the whole contracted block
(ab|cd) of a shell quartet in FP64 (or FP32 for the mixed form), the way the
reference's i2e_* kernels do (s_sp_l_terms.f90, s_p_d_terms.f90,
s_d_l_terms.f90), but with a Head-Gordon-Pople organisation:

  * per primitive quartet: Boys F_m(T) (m = 0..L) -> Obara-Saika vertical
    recurrence to [e0|f0]^(0) for e on A and f on C;
  * weighted contraction into per-sub-type accumulators -- an sp (L) shell is
    an s sub-shell with weight 1 and a p sub-shell with weight djkl (the p/s
    coefficient ratio, spread_basis.f90:149-151); S, P and D shells have one
    sub-shell whose coefficient is already in K_ab (precalc_kabs.f90:109);
  * after both primitive loops: horizontal recurrence on the ket
    [e0|c d) = [e0|c+1_i, d-1_i) + CD_i [e0|c, d-1_i), then on the bra;
  * Cartesian -> spherical transform for d shells (z2, xz, yz, xy, x2-y2;
    index_functions.f90:147-168).

Shell order inside a pair is "larger shell first" (D > L/P > S) so that the
horizontal recurrence always moves angular momentum from A to B and from C to
D.  The output block is out[((i*nB + j)*nC + k)*nD + l] in this order, each
shell's functions in the reference's component order (L: s,x,y,z).

Run as a script to regenerate ``generated/eri_classes.cuh``.
"""
from __future__ import annotations

import itertools
import math
import os
import sys
from typing import Dict, List, Tuple

# shell kinds in the GPU pair order: index used in pair-type codes
KINDS = ["S", "L", "D", "P"]
NFUNC = {"S": 1, "L": 4, "D": 5, "P": 3}
LMAX = {"S": 0, "L": 1, "D": 2, "P": 1}
# sub-shells: (angular momentum, weighted-by-ratio)
SUBS = {"S": [(0, False)], "L": [(0, False), (1, True)], "D": [(2, False)], "P": [(1, False)]}

# GPU pair types (larger shell first) and the quartet classes over {S,L,D}
PAIR_TYPES = [("S", "S"), ("L", "S"), ("L", "L"), ("D", "S"), ("D", "L"), ("D", "D")]
PAIR_NAMES = ["".join(p) for p in PAIR_TYPES]


def class_list():
    out = []
    for i in range(len(PAIR_TYPES)):
        for j in range(i, len(PAIR_TYPES)):
            out.append((i, j))
    return out


def carts(l: int) -> List[Tuple[int, int, int]]:
    """Cartesian monomials of degree l in the reference's order (indexps)."""
    out = []
    for i in range(l + 1):
        lx = l - i
        for n in range(i + 1):
            out.append((lx, i - n, n))
    return out


def add(a, i, d=1):
    t = list(a)
    t[i] += d
    return tuple(t)


Z3 = (0, 0, 0)
R3 = math.sqrt(3.0)
# matharmond rows: spherical (z2,xz,yz,xy,x2-y2) from Cartesian (xx,xy,xz,yy,yz,zz)
HARM = [[(-0.5, 0), (-0.5, 3), (1.0, 5)],
        [(R3, 2)],
        [(R3, 4)],
        [(R3, 1)],
        [(R3 / 2, 0), (-R3 / 2, 3)]]


class Emitter:
    def __init__(self, ftype: str):
        self.lines: List[str] = []
        self.n = 0
        self.ft = ftype

    def tmp(self, expr: str, prefix="t") -> str:
        self.n += 1
        name = f"{prefix}{self.n}"
        self.lines.append(f"    const {self.ft} {name} = {expr};")
        return name

    def raw(self, s: str):
        self.lines.append(s)


def fmt_coef(c: float, ft: str) -> str:
    s = repr(float(c))
    return s if ft == "double" else s + "f"


class VRR:
    """Obara-Saika vertical recurrence for [e0|f0]^(m), memoised."""

    def __init__(self, em: Emitter, order: str):
        self.em = em
        self.order = order
        self.nodes: Dict[Tuple, str] = {}
        self.nops = 0

    def get(self, e, f, m) -> str:
        key = (e, f, m)
        if key in self.nodes:
            return self.nodes[key]
        if e == Z3 and f == Z3:
            name = f"B{m}"
            self.nodes[key] = name
            return name
        if self.order == "bra":
            side = "bra" if sum(e) > 0 else "ket"
        else:
            side = "ket" if sum(f) > 0 else "bra"
        terms = []
        if side == "bra":
            i = max(range(3), key=lambda k: (e[k], -k))
            e1 = add(e, i, -1)
            terms.append(f"PA{i}*{self.get(e1, f, m)}")
            terms.append(f"WP{i}*{self.get(e1, f, m + 1)}")
            if e1[i] > 0:
                e2 = add(e1, i, -1)
                terms.append(f"h2p{e1[i]}*({self.get(e2, f, m)} - rp*{self.get(e2, f, m + 1)})")
            if f[i] > 0:
                f1 = add(f, i, -1)
                terms.append(f"h2pq{f[i]}*{self.get(e1, f1, m + 1)}")
        else:
            i = max(range(3), key=lambda k: (f[k], -k))
            f1 = add(f, i, -1)
            terms.append(f"QC{i}*{self.get(e, f1, m)}")
            terms.append(f"WQ{i}*{self.get(e, f1, m + 1)}")
            if f1[i] > 0:
                f2 = add(f1, i, -1)
                terms.append(f"h2q{f1[i]}*({self.get(e, f2, m)} - rq*{self.get(e, f2, m + 1)})")
            if e[i] > 0:
                e1 = add(e, i, -1)
                terms.append(f"h2pq{e[i]}*{self.get(e1, f, m + 1)}")
        self.nops += len(terms)
        name = self.em.tmp(" + ".join(terms), "v")
        self.nodes[key] = name
        return name


def sub_combos(t1: str, t2: str):
    """Sub-shell combinations of a pair: list of (l1, l2, weight-expression)."""
    out = []
    for (l1, w1), (l2, w2) in itertools.product(SUBS[t1], SUBS[t2]):
        w = []
        if w1:
            w.append("1")
        if w2:
            w.append("2")
        out.append((l1, l2, tuple(w)))
    return out


def comps(t: str):
    """Function list of a shell: (sub index, cartesian or spherical tag)."""
    if t == "S":
        return [(0, Z3)]
    if t == "P":
        return [(0, c) for c in carts(1)]
    if t == "L":
        return [(0, Z3)] + [(1, c) for c in carts(1)]
    return [(0, c) for c in carts(2)]  # D: Cartesian, transformed at the end


class ClassGen:
    def __init__(self, bra: Tuple[str, str], ket: Tuple[str, str], ftype="double", suffix=""):
        self.A, self.B = bra
        self.C, self.D = ket
        self.ft = ftype
        self.suffix = suffix
        self.L = LMAX[self.A] + LMAX[self.B] + LMAX[self.C] + LMAX[self.D]
        self.bra_combos = sub_combos(self.A, self.B)
        self.ket_combos = sub_combos(self.C, self.D)

    @property
    def name(self):
        return f"eri_{self.A}{self.B}_{self.C}{self.D}{self.suffix}"

    @property
    def nout(self):
        return NFUNC[self.A] * NFUNC[self.B] * NFUNC[self.C] * NFUNC[self.D]

    def targets(self):
        t = set()
        for (la, lb, _) in self.bra_combos:
            for (lc, ld, _) in self.ket_combos:
                for de in range(la, la + lb + 1):
                    for df in range(lc, lc + ld + 1):
                        for e in carts(de):
                            for f in carts(df):
                                t.add((e, f))
        return sorted(t)

    def gen_vrr(self, order):
        em = Emitter(self.ft)
        v = VRR(em, order)
        for (e, f) in self.targets():
            v.get(e, f, 0)
        return em, v

    def emit(self) -> str:
        ft = self.ft
        dbl = ft == "double"
        # choose the cheaper VRR order
        em_b, v_b = self.gen_vrr("bra")
        em_k, v_k = self.gen_vrr("ket")
        em, vrr = (em_b, v_b) if v_b.nops <= v_k.nops else (em_k, v_k)
        L = self.L
        # FLOP model (an FMA counts 2): per primitive quartet the set-up (~40),
        # Boys (Taylor 7 FMA + 2 per downward step), every VRR term (one FMA,
        # plus one for each (x - rho/p y) bracket) and every accumulation FMA;
        # per contracted quartet the HRR/spherical adds and the J/K scatter
        # (6 FMA per function quartet).
        nbracket = sum(line.count(" - r") for line in em.lines)
        nacc = sum(len(carts(de)) * len(carts(df))
                   for (la, lb, _) in self.bra_combos for (lc, ld, _) in self.ket_combos
                   for de in range(la, la + lb + 1) for df in range(lc, lc + ld + 1))
        self.flops_prim = 40 + 14 + 4 * L + 2 * vrr.nops + 2 * nbracket + 2 * nacc
        self.nvrr = vrr.nops
        out = []
        w = out.append
        w(f"// class ({self.A}{self.B}|{self.C}{self.D}): L={L}, {self.nout} functions, "
          f"VRR {vrr.nops} terms ({vrr.order}-first)")
        w(f"__device__ __forceinline__ void {self.name}(const GPair& bra, const GPair& ket,")
        w(f"    const GPrim* __restrict__ prims, const {ft}* __restrict__ btab, {ft}* __restrict__ out)")
        w("{")
        # accumulators
        acc = {}
        for bi, (la, lb, _) in enumerate(self.bra_combos):
            for ki, (lc, ld, _) in enumerate(self.ket_combos):
                for de in range(la, la + lb + 1):
                    for df in range(lc, lc + ld + 1):
                        for e in carts(de):
                            for f in carts(df):
                                nm = f"a{bi}{ki}_{''.join(map(str, e))}_{''.join(map(str, f))}"
                                acc[(bi, ki, e, f)] = nm
        w(f"    {ft} " + ", ".join(f"{n} = 0" for n in acc.values()) + ";")
        cv = (lambda s: s) if dbl else (lambda s: f"(float)({s})")
        w(f"    const double Ax = bra.A[0], Ay = bra.A[1], Az = bra.A[2];")
        w(f"    const double Cx = ket.A[0], Cy = ket.A[1], Cz = ket.A[2];")
        w("    for (int ib = 0; ib < bra.np; ++ib) {")
        w("        const GPrim pb = prims[bra.p0 + ib];")
        w(f"        const {ft} p = {cv('pb.p')};")
        w(f"        const {ft} PA0 = {cv('pb.P[0] - Ax')}, PA1 = {cv('pb.P[1] - Ay')}, PA2 = {cv('pb.P[2] - Az')};")
        # bra combo weights
        for bi, (_, _, wt) in enumerate(self.bra_combos):
            expr = " * ".join(cv(f"pb.w{x}") for x in wt) if wt else "1"
            w(f"        const {ft} wb{bi} = {expr};")
        w("        for (int ik = 0; ik < ket.np; ++ik) {")
        w("            const GPrim pk = prims[ket.p0 + ik];")
        w(f"            const {ft} q = {cv('pk.p')};")
        one = "1.0" if dbl else "1.0f"
        half = "0.5" if dbl else "0.5f"
        w(f"            const {ft} opq = {one} / (p + q);")
        w(f"            const {ft} rho = p * q * opq;")
        if dbl:
            w("            const double PQ0 = pb.P[0] - pk.P[0], PQ1 = pb.P[1] - pk.P[1], PQ2 = pb.P[2] - pk.P[2];")
        else:
            w("            const float PQ0 = (float)(pb.P[0] - pk.P[0]), PQ1 = (float)(pb.P[1] - pk.P[1]), PQ2 = (float)(pb.P[2] - pk.P[2]);")
        w(f"            const {ft} T = rho * (PQ0 * PQ0 + PQ1 * PQ1 + PQ2 * PQ2);")
        w(f"            {ft} F[{L + 1}];")
        w(f"            boys_eval<{L}>(T, btab, F);")
        if dbl:
            w("            const double pref = pb.K * pk.K * sqrt(opq);")
        else:
            w("            const float pref = (float)(pb.K * pk.K) * sqrtf(opq);")
        for m in range(L + 1):
            w(f"            const {ft} B{m} = pref * F[{m}];")
        if L > 0:
            # W - P = -q/(p+q) * (P - Q) ; W - Q = p/(p+q) * (P - Q)
            w(f"            const {ft} qo = q * opq, po = p * opq;")
            w(f"            const {ft} WP0 = -qo * PQ0, WP1 = -qo * PQ1, WP2 = -qo * PQ2;")
            w(f"            const {ft} WQ0 = po * PQ0, WQ1 = po * PQ1, WQ2 = po * PQ2;")
            if dbl:
                w("            const double QC0 = pk.P[0] - Cx, QC1 = pk.P[1] - Cy, QC2 = pk.P[2] - Cz;")
            else:
                w("            const float QC0 = (float)(pk.P[0] - Cx), QC1 = (float)(pk.P[1] - Cy), QC2 = (float)(pk.P[2] - Cz);")
            w(f"            const {ft} h2p1 = {half} / p, rp = rho / p;")
            w(f"            const {ft} h2q1 = {half} / q, rq = rho / q;")
            w(f"            const {ft} h2pq1 = {half} * opq;")
            for n in range(2, 5):
                w(f"            const {ft} h2p{n} = {n} * h2p1, h2q{n} = {n} * h2q1, h2pq{n} = {n} * h2pq1;")
        for ki, (_, _, wt) in enumerate(self.ket_combos):
            expr = " * ".join(cv(f"pk.w{x}") for x in wt) if wt else "1"
            w(f"            const {ft} wk{ki} = {expr};")
        for line in em.lines:
            w("        " + line)
        # accumulate
        for (bi, ki, e, f), nm in acc.items():
            src = vrr.nodes[(e, f, 0)]
            wexp = []
            if self.bra_combos[bi][2]:
                wexp.append(f"wb{bi}")
            if self.ket_combos[ki][2]:
                wexp.append(f"wk{ki}")
            if wexp:
                w(f"            {nm} += {' * '.join(wexp)} * {src};")
            else:
                w(f"            {nm} += {src};")
        w("        }")
        w("    }")
        # HRR
        hem = Emitter(ft)
        memo = {}
        w(f"    const {ft} AB0 = {cv('bra.A[0] - bra.B[0]')}, AB1 = {cv('bra.A[1] - bra.B[1]')}, AB2 = {cv('bra.A[2] - bra.B[2]')};")
        w(f"    const {ft} CD0 = {cv('ket.A[0] - ket.B[0]')}, CD1 = {cv('ket.A[1] - ket.B[1]')}, CD2 = {cv('ket.A[2] - ket.B[2]')};")

        def ket_hrr(bi, ki, e, c, d):
            key = ("k", bi, ki, e, c, d)
            if key in memo:
                return memo[key]
            if d == Z3:
                r = acc[(bi, ki, e, c)]
            else:
                i = max(range(3), key=lambda k: (d[k], -k))
                d1 = add(d, i, -1)
                x = ket_hrr(bi, ki, e, add(c, i), d1)
                y = ket_hrr(bi, ki, e, c, d1)
                r = hem.tmp(f"{x} + CD{i}*{y}", "h")
            memo[key] = r
            return r

        def bra_hrr(bi, ki, a, b, c, d):
            key = ("b", bi, ki, a, b, c, d)
            if key in memo:
                return memo[key]
            if b == Z3:
                r = ket_hrr(bi, ki, a, c, d)
            else:
                i = max(range(3), key=lambda k: (b[k], -k))
                b1 = add(b, i, -1)
                x = bra_hrr(bi, ki, add(a, i), b1, c, d)
                y = bra_hrr(bi, ki, a, b1, c, d)
                r = hem.tmp(f"{x} + AB{i}*{y}", "h")
            memo[key] = r
            return r

        # Cartesian results per component tuple
        cart = {}
        CA, CB, CC, CDc = comps(self.A), comps(self.B), comps(self.C), comps(self.D)
        for ia, (sa, ca) in enumerate(CA):
            for ib, (sb, cb) in enumerate(CB):
                bi = self.bra_combos.index(next(x for x in self.bra_combos if x[0] == SUBS[self.A][sa][0] and x[1] == SUBS[self.B][sb][0]))
                for ic, (sc, cc) in enumerate(CC):
                    for id_, (sd, cd) in enumerate(CDc):
                        ki = self.ket_combos.index(next(x for x in self.ket_combos if x[0] == SUBS[self.C][sc][0] and x[1] == SUBS[self.D][sd][0]))
                        cart[(ia, ib, ic, id_)] = bra_hrr(bi, ki, ca, cb, cc, cd)
        for line in hem.lines:
            w(line)
        self.nhrr = len(hem.lines)
        # spherical transform of d shells, centre by centre
        dims = [len(CA), len(CB), len(CC), len(CDc)]
        types = [self.A, self.B, self.C, self.D]
        sem = Emitter(ft)
        cur = cart
        for ax in range(4):
            if types[ax] != "D":
                continue
            nxt = {}
            rng = [range(d) for d in dims]
            rng[ax] = range(5)
            for idx in itertools.product(*rng):
                terms = []
                for coef, cc in HARM[idx[ax]]:
                    src = list(idx)
                    src[ax] = cc
                    v = cur[tuple(src)]
                    terms.append(v if coef == 1.0 else f"{fmt_coef(coef, ft)}*{v}")
                nxt[idx] = sem.tmp(" + ".join(terms), "s")
            dims[ax] = 5
            cur = nxt
        for line in sem.lines:
            w(line)
        nsph = sum(l.count("+") + 1 for l in sem.lines)
        self.flops_quartet = 2 * self.nhrr + 2 * nsph + 12 * self.nout
        n = 0
        for idx in itertools.product(*[range(d) for d in dims]):
            w(f"    out[{n}] = {cur[idx]};")
            n += 1
        assert n == self.nout
        w("}")
        return "\n".join(out)


CLASS_TU = """// GENERATED by gen_eri.py -- do not edit.
// Kernels of quartet class ({A}{B}|{C}{D}).
#include "../common.cuh"

namespace hfgpu {{
{body}

#define HF_THIS_CLASS HF_CLASS_TRAITS({ci}, {bi}, {ki}, {A}{B}_{C}{D}, {nout}, {L})
HF_THIS_CLASS
#undef HF_THIS_CLASS

void register_class_{ci}(ClassKernels* k) {{
    k->nd64 = k_nondiag<Cls_{A}{B}_{C}{D}, false>;
    k->nd32 = k_nondiag<Cls_{A}{B}_{C}{D}, true>;
{diag}    k->bi = {bi};
    k->ki = {ki};
    k->L = {L};
    k->nout = {nout};
}}

}}  // namespace hfgpu
"""


def main(outdir: str):
    os.makedirs(outdir, exist_ok=True)
    names = []
    flops = {}
    for ci, (bi, ki) in enumerate(class_list()):
        g = ClassGen(PAIR_TYPES[bi], PAIR_TYPES[ki], "double")
        g32 = ClassGen(PAIR_TYPES[bi], PAIR_TYPES[ki], "float", suffix="_f32")
        body = g.emit() + "\n\n" + g32.emit()
        diag = ""
        if bi == ki:
            diag = (f"    k->diag0 = k_diag<Cls_{g.A}{g.B}_{g.C}{g.D}, 0>;\n"
                    f"    k->diag1 = k_diag<Cls_{g.A}{g.B}_{g.C}{g.D}, 1>;\n")
        else:
            diag = "    k->diag0 = nullptr;\n    k->diag1 = nullptr;\n"
        flops[ci] = {"name": f"{g.A}{g.B}|{g.C}{g.D}", "L": g.L, "nout": g.nout,
                     "flops_prim": g.flops_prim, "flops_quartet": g.flops_quartet,
                     "vrr_terms": g.nvrr, "hrr_terms": g.nhrr}
        text = CLASS_TU.format(A=g.A, B=g.B, C=g.C, D=g.D, body=body, ci=ci, bi=bi, ki=ki,
                               nout=g.nout, L=g.L, diag=diag)
        fn = os.path.join(outdir, f"cls_{ci:02d}_{g.A}{g.B}_{g.C}{g.D}.cu")
        new = text
        if not os.path.exists(fn) or open(fn).read() != new:
            with open(fn, "w") as fh:
                fh.write(new)
        names.append(fn)
    import json
    fl = os.path.join(outdir, "class_flops.json")
    txt = json.dumps(flops, indent=1)
    if not os.path.exists(fl) or open(fl).read() != txt:
        with open(fl, "w") as fh:
            fh.write(txt)
    return names


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)), "generated"))
