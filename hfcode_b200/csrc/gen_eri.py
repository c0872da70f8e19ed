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
import json
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
# GPU pair types, larger shell first (D > L > P > S); the four with pure p
# shells come last so the classes of the {s, l, d} bases keep indices 0..20
PAIR_TYPES = [("S", "S"), ("L", "S"), ("L", "L"), ("D", "S"), ("D", "L"), ("D", "D"),
              ("P", "S"), ("L", "P"), ("P", "P"), ("D", "P")]
N_SLD_TYPES = 6
PAIR_NAMES = ["".join(p) for p in PAIR_TYPES]


def class_list():
    """Quartet classes (bra type <= ket type): the 21 classes over the
    {s, l, d} pair types first, then every class with a pure-p pair type."""
    n = len(PAIR_TYPES)
    out = [(i, j) for i in range(N_SLD_TYPES) for j in range(i, N_SLD_TYPES)]
    out += [(i, j) for i in range(n) for j in range(i, n) if j >= N_SLD_TYPES]
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
                terms.append(f"h2pq{e[i]}*{self.get(e1, f1, m + 1)}")
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
    """Code generator of one quartet class (A B|C D), GPU shell order."""

    def __init__(self, bra: Tuple[str, str], ket: Tuple[str, str], ftype="double", suffix=""):
        self.A, self.B = bra
        self.C, self.D = ket
        self.ft = ftype
        self.suffix = suffix
        self.L = LMAX[self.A] + LMAX[self.B] + LMAX[self.C] + LMAX[self.D]
        self.bra_combos = sub_combos(self.A, self.B)
        self.ket_combos = sub_combos(self.C, self.D)
        self.types = [self.A, self.B, self.C, self.D]
        self.cl = [comps(t) for t in self.types]
        self.nf = [NFUNC[t] for t in self.types]
        self.outputs = list(itertools.product(*[range(n) for n in self.nf]))
        self._leaf_cache: Dict[Tuple, frozenset] = {}

    @property
    def tag(self):
        return f"{self.A}{self.B}_{self.C}{self.D}"

    @property
    def name(self):
        return f"eri_{self.tag}{self.suffix}"

    @property
    def nout(self):
        return len(self.outputs)

    # ---------------------------------------------------------------- deps
    def cart_terms(self, o):
        """Output function (i,j,k,l) as sum of coef * Cartesian (ca,cb,cc,cd)."""
        per = []
        for ax, t in enumerate(self.types):
            if t == "D":
                per.append(HARM[o[ax]])
            else:
                per.append([(1.0, o[ax])])
        out = []
        for combo in itertools.product(*per):
            c = 1.0
            idx = []
            for coef, ci in combo:
                c *= coef
                idx.append(ci)
            out.append((c, tuple(idx)))
        return out

    def combo_of(self, cart4):
        sa, sb, sc, sd = (self.cl[ax][cart4[ax]][0] for ax in range(4))
        la, lb = SUBS[self.A][sa][0], SUBS[self.B][sb][0]
        lc, ld = SUBS[self.C][sc][0], SUBS[self.D][sd][0]
        bi = next(i for i, x in enumerate(self.bra_combos) if x[0] == la and x[1] == lb)
        ki = next(i for i, x in enumerate(self.ket_combos) if x[0] == lc and x[1] == ld)
        return bi, ki

    def leaves(self, cart4) -> frozenset:
        """Accumulator keys (bi, ki, e, f) the HRR of one Cartesian quartet reads."""
        if cart4 in self._leaf_cache:
            return self._leaf_cache[cart4]
        bi, ki = self.combo_of(cart4)
        a, b, c, d = (self.cl[ax][cart4[ax]][1] for ax in range(4))
        out = set()

        def ket(e, c, d):
            if d == Z3:
                out.add((bi, ki, e, c))
                return
            i = max(range(3), key=lambda k: (d[k], -k))
            d1 = add(d, i, -1)
            ket(e, add(c, i), d1)
            ket(e, c, d1)

        def bra(a, b):
            if b == Z3:
                ket(a, c, d)
                return
            i = max(range(3), key=lambda k: (b[k], -k))
            b1 = add(b, i, -1)
            bra(add(a, i), b1)
            bra(a, b1)

        bra(a, b)
        r = frozenset(out)
        self._leaf_cache[cart4] = r
        return r

    def out_leaves(self, o):
        s = set()
        for _, c4 in self.cart_terms(o):
            s |= self.leaves(c4)
        return s

    def partition(self, acc_max: int, out_max: int):
        """Greedy split of the outputs (flat order) into roles whose
        accumulator and output counts fit the register budget."""
        groups, cur, cur_acc = [], [], set()
        for n, o in enumerate(self.outputs):
            lv = self.out_leaves(o)
            if cur and (len(cur_acc | lv) > acc_max or len(cur) >= out_max):
                groups.append(cur)
                cur, cur_acc = [], set()
            cur.append(n)
            cur_acc |= lv
        if cur:
            groups.append(cur)
        return groups

    # ---------------------------------------------------------------- emit
    def _vrr_block(self, keys):
        """Primitive loops: Boys, VRR and the weighted accumulation of the
        accumulator keys.  Returns (lines, acc name map, stats)."""
        ft = self.ft
        dbl = ft == "double"
        L = self.L
        cv = (lambda s: s) if dbl else (lambda s: f"(float)({s})")
        targets = sorted({(e, f) for (_, _, e, f) in keys})

        def gen_vrr(order):
            em = Emitter(ft)
            v = VRR(em, order)
            for (e, f) in targets:
                v.get(e, f, 0)
            return em, v

        em_b, v_b = gen_vrr("bra")
        em_k, v_k = gen_vrr("ket")
        em, vrr = (em_b, v_b) if v_b.nops <= v_k.nops else (em_k, v_k)
        acc = {}
        for key in sorted(keys, key=lambda k: (k[0], k[1], sum(k[2]), k[2], sum(k[3]), k[3])):
            bi, ki, e, f = key
            acc[key] = f"a{bi}{ki}_{''.join(map(str, e))}_{''.join(map(str, f))}"
        out = []
        w = out.append
        w(f"    {ft} " + ", ".join(f"{n} = 0" for n in acc.values()) + ";")
        w("    const double Ax = bra.A[0], Ay = bra.A[1], Az = bra.A[2];")
        w("    const double Cx = ket.A[0], Cy = ket.A[1], Cz = ket.A[2];")
        w("    for (int ib = 0; ib < bra.np; ++ib) {")
        w("        const GPrim pb = load_prim(prims, bra.p0 + ib * bra.ps);")
        w(f"        const {ft} p = {cv('pb.p')};")
        w(f"        const {ft} PA0 = {cv('pb.P[0] - Ax')}, PA1 = {cv('pb.P[1] - Ay')}, PA2 = {cv('pb.P[2] - Az')};")
        if L > 0:
            w(f"        const {ft} h2p1 = {cv('pb.pad')};  // 1/(2p), precomputed per primitive pair")
        used_b = sorted({k[0] for k in acc})
        used_k = sorted({k[1] for k in acc})
        for bi in used_b:
            wt = self.bra_combos[bi][2]
            expr = " * ".join(cv(f"pb.w{x}") for x in wt) if wt else "1"
            w(f"        const {ft} wb{bi} = {expr};")
        w("        for (int ik = 0; ik < ket.np; ++ik) {")
        w("            const GPrim pk = load_prim(prims, ket.p0 + ik * ket.ps);")
        w(f"            const {ft} q = {cv('pk.p')};")
        one = "1.0" if dbl else "1.0f"
        half = "0.5" if dbl else "0.5f"
        # one reciprocal square root per primitive quartet gives both
        # 1/(p+q) and the sqrt(1/(p+q)) of the prefactor
        w(f"            const {ft} rs = {'rsqrt' if dbl else 'rsqrtf'}(p + q);")
        w(f"            const {ft} opq = rs * rs;")
        w(f"            const {ft} rho = p * q * opq;")
        if dbl:
            w("            const double PQ0 = pb.P[0] - pk.P[0], PQ1 = pb.P[1] - pk.P[1], PQ2 = pb.P[2] - pk.P[2];")
        else:
            w("            const float PQ0 = (float)(pb.P[0] - pk.P[0]), PQ1 = (float)(pb.P[1] - pk.P[1]), "
              "PQ2 = (float)(pb.P[2] - pk.P[2]);")
        w(f"            const {ft} T = rho * (PQ0 * PQ0 + PQ1 * PQ1 + PQ2 * PQ2);")
        w(f"            {ft} F[{L + 1}];")
        w(f"            boys_eval<{L}>(T, btab, F);")
        if dbl:
            w("            const double pref = pb.K * pk.K * rs;")
        else:
            w("            const float pref = (float)(pb.K * pk.K) * rs;")
        for m in range(L + 1):
            w(f"            const {ft} B{m} = pref * F[{m}];")
        if L > 0:
            w(f"            const {ft} qo = q * opq, po = p * opq;")
            w(f"            const {ft} WP0 = -qo * PQ0, WP1 = -qo * PQ1, WP2 = -qo * PQ2;")
            w(f"            const {ft} WQ0 = po * PQ0, WQ1 = po * PQ1, WQ2 = po * PQ2;")
            if dbl:
                w("            const double QC0 = pk.P[0] - Cx, QC1 = pk.P[1] - Cy, QC2 = pk.P[2] - Cz;")
            else:
                w("            const float QC0 = (float)(pk.P[0] - Cx), QC1 = (float)(pk.P[1] - Cy), "
                  "QC2 = (float)(pk.P[2] - Cz);")
            w(f"            const {ft} rp = qo, rq = po;  // rho/p = q/(p+q), rho/q = p/(p+q)")
            w(f"            const {ft} h2q1 = {cv('pk.pad')};  // 1/(2q), precomputed per primitive pair")
            w(f"            const {ft} h2pq1 = {half} * opq;")
            for n in range(2, 5):
                w(f"            const {ft} h2p{n} = {n} * h2p1, h2q{n} = {n} * h2q1, h2pq{n} = {n} * h2pq1;")
        for ki in used_k:
            wt = self.ket_combos[ki][2]
            expr = " * ".join(cv(f"pk.w{x}") for x in wt) if wt else "1"
            w(f"            const {ft} wk{ki} = {expr};")
        for line in em.lines:
            w("        " + line)
        for (bi, ki, e, f), nm in acc.items():
            src = vrr.nodes[(e, f, 0)]
            wexp = []
            if self.bra_combos[bi][2]:
                wexp.append(f"wb{bi}")
            if self.ket_combos[ki][2]:
                wexp.append(f"wk{ki}")
            w(f"            {nm} += {' * '.join(wexp + [src])};")
        w("        }")
        w("    }")
        nbracket = sum(line.count(" - r") for line in em.lines)
        return out, acc, {"vrr": vrr.nops, "bracket": nbracket, "acc": len(acc), "order": vrr.order}

    def _hrr_block(self, outs, leaf, ft, store=None):
        """HRR on ket and bra plus the spherical transform for `outs`;
        leaf(key) names the contracted accumulator, or returns (name, line)
        to have the line (its load) emitted where it is first used.  With
        `store`, store(r, expr) is emitted right after output r's terms, so
        each output leaves the registers as soon as it is formed.  Returns
        (lines, value expressions per output, stats)."""
        cv = (lambda s: s) if ft == "double" else (lambda s: f"(float)({s})")
        lines = [f"    const {ft} AB0 = {cv('bra.A[0] - bra.B[0]')}, AB1 = {cv('bra.A[1] - bra.B[1]')}, "
                 f"AB2 = {cv('bra.A[2] - bra.B[2]')};",
                 f"    const {ft} CD0 = {cv('ket.A[0] - ket.B[0]')}, CD1 = {cv('ket.A[1] - ket.B[1]')}, "
                 f"CD2 = {cv('ket.A[2] - ket.B[2]')};"]
        hem = Emitter(ft)
        memo = {}

        def ket_hrr(bi, ki, e, c, d):
            key = ("k", bi, ki, e, c, d)
            if key in memo:
                return memo[key]
            if d == Z3:
                r = leaf((bi, ki, e, c))
                if isinstance(r, tuple):
                    r, ln = r
                    if ln:
                        hem.raw(ln)
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

        vals = []
        nsph = 0
        for n in outs:
            terms = []
            for coef, c4 in self.cart_terms(self.outputs[n]):
                bi, ki = self.combo_of(c4)
                a, b, c, d = (self.cl[ax][c4[ax]][1] for ax in range(4))
                v = bra_hrr(bi, ki, a, b, c, d)
                terms.append(v if coef == 1.0 else f"{fmt_coef(coef, ft)}*{v}")
            nsph += len(terms) - 1
            vals.append(" + ".join(terms))
            if store is not None:
                hem.raw(store(len(vals) - 1, vals[-1]))
        nh = sum(1 for ln in hem.lines if ln.lstrip().startswith(f"const {ft} h"))
        lines += hem.lines
        return lines, vals, {"hrr": nh, "sph": nsph}

    def needed_keys(self, outs):
        keys = set()
        for n in outs:
            keys |= self.out_leaves(self.outputs[n])
        return keys

    def all_keys(self):
        return self.needed_keys(range(self.nout))

    def emit_role(self, fname: str, outs: List[int]):
        """Device function computing the outputs `outs` (flat indices) into
        out[0..len(outs)).  Returns (code, stats)."""
        ft = self.ft
        vlines, acc, vst = self._vrr_block(self.needed_keys(outs))
        hlines, vals, hst = self._hrr_block(outs, lambda k: acc[k], ft)
        out = [f"// ({self.A}{self.B}|{self.C}{self.D}) outputs {outs[0]}..{outs[-1]} ({len(outs)}): L={self.L}, "
               f"{vst['acc']} accumulators, VRR {vst['vrr']} terms ({vst['order']}-first)",
               f"__device__ __forceinline__ void {fname}(const GPair& bra, const GPair& ket,",
               f"    const PrimSoA& prims, const {ft}* __restrict__ btab, {ft}* __restrict__ out)",
               "{"]
        out += vlines + hlines
        out += [f"    out[{r}] = {v};" for r, v in enumerate(vals)]
        out.append("}")
        return "\n".join(out), {**vst, **hst}

    def emit_acc_role(self, fname: str, keys: List[Tuple]):
        """Stage-A device function: the contracted accumulators `keys`,
        written to dst[k * stride] (k = position in `keys`)."""
        ft = self.ft
        vlines, acc, vst = self._vrr_block(set(keys))
        out = [f"// ({self.A}{self.B}|{self.C}{self.D}) accumulators ({len(keys)}): VRR {vst['vrr']} terms "
               f"({vst['order']}-first)",
               f"__device__ __forceinline__ void {fname}(const GPair& bra, const GPair& ket,",
               f"    const PrimSoA& prims, const {ft}* __restrict__ btab, {ft}* __restrict__ dst, "
               f"size_t stride)",
               "{"]
        out += vlines
        out += [f"    dst[{k} * stride] = {acc[key]};" for k, key in enumerate(keys)]
        out.append("}")
        return "\n".join(out), vst

    def emit_hrr_role(self, fname: str, outs: List[int], keyidx: Dict[Tuple, int]):
        """Stage-B device function: outputs `outs` from the accumulators in
        src[keyidx[key] * stride], written to dst[r * stride]; returns
        max |value|.  Accumulators, arithmetic and outputs are in the
        generator's type (FP32 chunks keep FP32 throughout)."""
        ft = self.ft
        loaded = {}

        def leaf(key):
            # each accumulator is loaded where the recursion first needs it
            # and each output is stored as soon as it is formed: hoisting
            # every load to the top and every store to the end kept all of
            # them live at once and spilled the d-heavy roles
            if key not in loaded:
                nm = f"L{keyidx[key]}"
                loaded[key] = nm
                return nm, f"    const {ft} {nm} = __ldg(src + {keyidx[key]} * stride);"
            return loaded[key], None

        def store(r, v):
            return f"    {{ const {ft} v = {v}; dst[{r} * stride] = v; mx = fmax(mx, fabs((double)v)); }}"

        hlines, vals, hst = self._hrr_block(outs, leaf, ft, store)
        out = [f"// ({self.A}{self.B}|{self.C}{self.D}) outputs {outs[0]}..{outs[-1]} ({len(outs)}) from accumulators",
               f"__device__ __forceinline__ double {fname}(const GPair& bra, const GPair& ket,",
               f"    const {ft}* __restrict__ src, {ft}* __restrict__ dst, size_t stride)",
               "{",
               "    double mx = 0.0;"]
        out += hlines
        out.append("    return mx;")
        out.append("}")
        return "\n".join(out), hst

    def flop_model(self):
        """Algorithmic FLOPs of the class in its single-function formulation
        (an FMA counts 2): per primitive quartet the set-up (~40), Boys
        (Taylor 7 FMA + 2 per downward step), every VRR term (one FMA, plus
        one for each (x - rho/p y) bracket) and every accumulation FMA; per
        contracted quartet the HRR/spherical adds and the J/K scatter (6 FMA
        per function quartet)."""
        _, st = self.emit_role("_count", list(range(self.nout)))
        self.flops_prim = 40 + 14 + 4 * self.L + 2 * st["vrr"] + 2 * st["bracket"] + 2 * st["acc"]
        self.flops_quartet = 2 * st["hrr"] + 2 * st["sph"] + 12 * self.nout
        self.nvrr, self.nhrr = st["vrr"], st["hrr"]

    # ------------------------------------------------------------- scatter
    def emit_scatter(self, fname: str, outs: List[int]) -> str:
        """J/K scatter of the outputs `outs` with uniform weight s into the
        one-triangle buffer G (F += G + G^T later); P is column-major."""
        o4 = [self.outputs[n] for n in outs]
        lines = [f"template <typename E>",
                 f"__device__ __forceinline__ void {fname}(const E* __restrict__ e, double s, const GPair& bra, "
                 f"const GPair& ket, const double* __restrict__ P, double* __restrict__ G, int nb, bool jonly)",
                 "{",
                 "    const int a0 = bra.aoa, b0 = bra.aob, c0 = ket.aoa, d0 = ket.aob;",
                 "    const double s2 = 2.0 * s, hs = -0.5 * s;"]
        loaded = set()
        org = {"a": "a0", "b": "b0", "c": "c0", "d": "d0"}

        def pv(x, i, y, j):
            nm = f"p{x}{i}{y}{j}"
            if nm not in loaded:
                loaded.add(nm)
                lines.append(f"    const double {nm} = __ldg(P + ({org[x]} + {i}) + (size_t)({org[y]} + {j}) * nb);")
            return nm

        def block(rowx, rowi, colx, coli, px, pi, qx, qi, scale, tgt):
            groups: Dict[Tuple[int, int], List[Tuple[int, int]]] = {}
            for r, o in enumerate(o4):
                key = (o[rowi], o[coli])
                groups.setdefault(key, []).append((r, o))
            for (i, j), lst in groups.items():
                terms = [f"{pv(px, o[pi], qx, o[qi])} * (double)e[{r}]" for r, o in lst]
                lines.append(f"    atomicAdd(G + ({org[rowx]} + {i}) + (size_t)({org[colx]} + {j}) * nb, "
                             f"{scale} * ({' + '.join(terms)}));")

        # J_ab <- P_cd, J_cd <- P_ab
        block("a", 0, "b", 1, "c", 2, "d", 3, "s2", "J")
        block("c", 2, "d", 3, "a", 0, "b", 1, "s2", "J")
        lines.append("    if (jonly) return;")
        # K_ac <- P_bd, K_ad <- P_bc, K_bc <- P_ad, K_bd <- P_ac
        block("a", 0, "c", 2, "b", 1, "d", 3, "hs", "K")
        block("a", 0, "d", 3, "b", 1, "c", 2, "hs", "K")
        block("b", 1, "c", 2, "a", 0, "d", 3, "hs", "K")
        block("b", 1, "d", 3, "a", 0, "c", 2, "hs", "K")
        lines.append("}")
        return "\n".join(lines)


ACC_MAX = 64        # accumulators per output role (register budget)
OUT_MAX = 32        # outputs per output role
MAX_ROLES2 = 12     # beyond this, the class goes through the accumulator stage
ACC_GROUP = 48      # accumulators per stage-A role (d-heavy classes)
OUT_GROUP3 = 25     # outputs per stage-B role (d-heavy classes)
MAXR = 64           # role slots in ClassKernels

# Per-class shape overrides (measured on the device; see tuning.json beside
# this file): {"<tag>": {"acc_max": .., "out_max": .., "max_roles2": ..,
# "acc_group": .., "out_group3": .., "staged": true}}; "staged" keeps a
# one-role class on the staged path (outputs through scratch, staged scatter)
# instead of the direct one.  HFGPU_TUNING names another file.
_TUNING_FILE = os.environ.get("HFGPU_TUNING") or os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                              "tuning.json")


def class_params(tag: str) -> dict:
    prm = {"acc_max": ACC_MAX, "out_max": OUT_MAX, "max_roles2": MAX_ROLES2, "acc_group": ACC_GROUP,
           "out_group3": OUT_GROUP3}
    if os.path.exists(_TUNING_FILE):
        with open(_TUNING_FILE) as fh:
            prm.update(json.load(fh).get(tag, {}))
    prm.setdefault("acc_max32", 2 * prm["acc_max"])
    prm.setdefault("acc_group32", 2 * prm["acc_group"])
    prm.setdefault("out_max32", 2 * prm["out_max"])
    prm.setdefault("minb32", 2)  # blocks per SM of the FP32 output-role kernels (staged2)
    return prm


def acc_groups(g: "ClassGen", group: int = ACC_GROUP):
    """Partition of all accumulator keys into stage-A roles; the key order
    that minimises the summed VRR terms wins."""
    keys = list(g.all_keys())
    orders = {
        "ket": lambda k: (k[1], sum(k[3]), k[3], k[0], sum(k[2]), k[2]),
        "bra": lambda k: (k[0], sum(k[2]), k[2], k[1], sum(k[3]), k[3]),
        "f": lambda k: (sum(k[3]), k[3], k[1], k[0], sum(k[2]), k[2]),
        "e": lambda k: (sum(k[2]), k[2], k[0], k[1], sum(k[3]), k[3]),
    }
    best = None
    for name, fn in orders.items():
        ks = sorted(keys, key=fn)
        groups = [ks[i:i + group] for i in range(0, len(ks), group)]
        cost = sum(g._vrr_block(set(gr))[2]["vrr"] for gr in groups)
        if best is None or cost < best[0]:
            best = (cost, groups)
    return best[1]


def merged_kernel(kname: str, bodies: List[str], minb: int = 2) -> str:
    """All roles of one stage in one launch: block row blockIdx.y runs role
    blockIdx.y (every thread of a block runs the same role).  Used for small
    chunks, where one launch per role would leave most SMs idle and the
    launches themselves would set the time."""
    cases = "\n".join(f"        case {r}: {b}_body(a); break;" for r, b in enumerate(bodies))
    return f"""
__global__ void __launch_bounds__(RB_THREADS, {minb} * RB_SCALE) {kname}(StagedArgs a) {{
    switch (blockIdx.y) {{
{cases}
        default: break;
    }}
}}"""


def grouped_scatter_reg(NA: int, NB: int, NC: int, ND: int, prm: dict) -> str:
    """Registration of the grouped scatter (four lanes per quartet, lane g
    owning function g of a four-function bra shell: the first shell when it
    has four functions, else the second), or nullptr when neither has.
    scat_grouped64 / scat_grouped32 in the tuning table choose it by default
    for the FP64 / FP32 chunks of the class (measured per class)."""
    S = 0 if NA == 4 else 1 if NB == 4 else -1
    if S < 0:
        return ("    k->scatg = nullptr;\n    k->scatg32 = nullptr;\n"
                "    k->scatg_smem = 0;\n    k->scatg32_smem = 0;\n    k->grp64 = 0;\n    k->grp32 = 0;")
    NX = NB if S == 0 else NA
    return (f"    k->scatg = k_scatter_grouped<{NA}, {NB}, {NC}, {ND}, {S}>;\n"
            f"    k->scatg_smem = scatg_smem_bytes({NX}, {NC}, {ND}, 8);\n"
            f"    k->scatg32 = k_scatter_grouped<{NA}, {NB}, {NC}, {ND}, {S}, float>;\n"
            f"    k->scatg32_smem = scatg_smem_bytes({NX}, {NC}, {ND}, 4);\n"
            f"    k->grp64 = {int(bool(prm.get('scat_grouped64', False)))};\n"
            f"    k->grp32 = {int(bool(prm.get('scat_grouped32', False)))};")


def class_source(ci: int, bi: int, ki: int):
    """Header (device functions) and translation unit (kernels) of one
    quartet class; returns (cuh_text, cu_text, info).

    Three shapes:
      direct  one thread per quartet computes the whole block (k_nondiag);
      staged2 the outputs are split into roles, one kernel launch per role
              (uniform code per launch), each writing its outputs and their
              max to a scratch buffer; k_scatter_staged applies the
              post-screen and the J/K scatter;
      staged3 (d-heavy) stage-A roles write the contracted [e0|f0]
              accumulators to scratch, stage-B roles apply the HRR and the
              spherical transform to slices of the outputs, then the same
              scatter kernel."""
    g = ClassGen(PAIR_TYPES[bi], PAIR_TYPES[ki], "double")
    g32 = ClassGen(PAIR_TYPES[bi], PAIR_TYPES[ki], "float", suffix="_f32")
    g.flop_model()
    prm = class_params(g.tag)
    roles = g.partition(prm["acc_max"], prm["out_max"])
    funcs, kern = [], []
    reg = []
    NA, NB, NC, ND = g.nf
    info = {"name": f"{g.A}{g.B}|{g.C}{g.D}", "tag": g.tag, "L": g.L, "nout": g.nout,
            "flops_prim": g.flops_prim, "flops_quartet": g.flops_quartet,
            "vrr_terms": g.nvrr, "hrr_terms": g.nhrr}
    if len(roles) == 1 and not prm.get("staged", False):
        mode = "direct"
        code, _ = g.emit_role(g.name, roles[0])
        code32, _ = g32.emit_role(g32.name, roles[0])
        funcs += [code, code32]
        reg.append(f"    k->mode = 0;")
        reg.append(f"    k->nd64 = k_nondiag<Cls_{g.tag}, false>;")
        reg.append(f"    k->nd32 = k_nondiag<Cls_{g.tag}, true>;")
        reg.append(f"    k->nd_threads = ND_THREADS;\n    k->nd_qpb = ND_THREADS;")
        if bi == ki:
            reg.append(f"    k->diag0 = k_diag<Cls_{g.tag}, 0>;\n    k->diag1 = k_diag<Cls_{g.tag}, 1>;")
            reg.append(f"    k->dg_threads = ND_THREADS;\n    k->dg_ppb = ND_THREADS;")
        info.update(roles=1, role_sizes=[g.nout], role_outs=[roles[0]], acc_groups=[])
    elif len(roles) <= prm["max_roles2"]:
        mode = "staged2"
        # FP32 values take half the registers: the FP32 kernels use roles of
        # twice the size, so fewer of them repeat the primitive loop
        roles32 = g.partition(prm["acc_max32"], prm["out_max32"])

        def nroles_of(f32):  # rows of the role maxima of a chunk of this precision
            return len(roles32) if f32 else len(roles)

        def s2_kernel(kname, fname, outs, r, f32):
            real = "float" if f32 else "double"
            stores = "\n".join(f"    {{ const double v = (double)e[{i}]; out[{n} * TQ] = ({real})v; "
                               f"mx = fmax(mx, fabs(v)); }}" for i, n in enumerate(outs))
            tab = "a.boysf" if f32 else "a.boys"
            return f"""
__device__ __forceinline__ void {kname}_body(const StagedArgs& a) {{
    // Boys table of order L read through the L1 cache: with a few primitive
    // quartets per shell quartet, staging it in shared memory per block
    // costs more than the lookups it serves
    const {real}* __restrict__ sboys = {tab} + (size_t){g.L} * BOYS_BLK;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= staged_count(a)) return;
    const uint2 q = staged_quartet(a, t);
    const GPair bra = a.bra[q.x];
    const GPair ket = a.ket[q.y];
    {real} e[{len(outs)}];
    {fname}(bra, ket, a.prims, sboys, e);
    double mx = 0.0;
    // this quartet's column of the chunk's output tile (FP32 chunks keep FP32 rows)
    {real}* out = reinterpret_cast<{real}*>(a.out) + tcol(t, {g.nout});
{stores}
    a.mx[tcol(t, {nroles_of(f32)}) + {r} * TQ] = mx;
}}
__global__ void __launch_bounds__(RB_THREADS, {prm["minb32"] if f32 else 2} * RB_SCALE) {kname}(StagedArgs a) {{ {kname}_body(a); }}"""

        for r, outs in enumerate(roles):
            code, _ = g.emit_role(f"{g.name}_r{r}", outs)
            funcs.append(code)
            kern.append(s2_kernel(f"k_s2_{g.tag}_r{r}", f"eri_{g.tag}_r{r}", outs, r, False))
        for r, outs in enumerate(roles32):
            code32, _ = g32.emit_role(f"{g32.name}_r{r}", outs)
            funcs.append(code32)
            kern.append(s2_kernel(f"k_s2f_{g.tag}_r{r}", f"eri_{g.tag}_f32_r{r}", outs, r, True))
        kern.append(merged_kernel(f"k_s2m_{g.tag}", [f"k_s2_{g.tag}_r{r}" for r in range(len(roles))]))
        kern.append(merged_kernel(f"k_s2mf_{g.tag}", [f"k_s2f_{g.tag}_r{r}" for r in range(len(roles32))]))
        reg.append(f"    k->mb64 = k_s2m_{g.tag};\n    k->mb32 = k_s2mf_{g.tag};")
        reg.append(f"    k->mode = 1;\n    k->nacc = 0;\n    k->nrole_a = 0;\n    k->nrole_b = {len(roles)};\n"
                   f"    k->nrole_b32 = {len(roles32)};")
        for r in range(len(roles)):
            reg.append(f"    k->sb64[{r}] = k_s2_{g.tag}_r{r};")
        for r in range(len(roles32)):
            reg.append(f"    k->sb32[{r}] = k_s2f_{g.tag}_r{r};")
        reg.append(f"    k->scat = k_scatter_staged<{NA}, {NB}, {NC}, {ND}>;\n"
                   f"    k->scat_smem = scat_smem_bytes({NA}, {NB}, {NC}, {ND});\n"
                   f"    k->scat32 = k_scatter_staged<{NA}, {NB}, {NC}, {ND}, float>;\n"
                   f"    k->scat32_smem = scat_smem_bytes({NA}, {NB}, {NC}, {ND}, 4);")
        reg.append(grouped_scatter_reg(NA, NB, NC, ND, prm))
        if bi == ki:
            reg.append(f"    k->diag0 = nullptr;\n    k->diag1 = nullptr;")
            reg.append(f"    k->dscat0 = k_scatter_diag<{NA}, {NB}, 0>;\n    k->dscat1 = k_scatter_diag<{NA}, {NB}, 1>;")
        info["role_outs32"] = roles32
        info.update(roles=len(roles), role_sizes=[len(x) for x in roles], role_outs=roles, acc_groups=[])
    else:
        mode = "staged3"
        groups = acc_groups(g, prm["acc_group"])
        keyidx = {}
        for gr in groups:
            for key in gr:
                keyidx[key] = len(keyidx)
        # FP32 values take half the registers: the FP32 stage-A roles take
        # acc_group32 accumulators (consecutive FP64 groups merged), so fewer
        # of them repeat the primitive loop; the accumulator layout is the same
        per32 = max(1, prm["acc_group32"] // prm["acc_group"])
        groups32 = [sum(groups[i:i + per32], []) for i in range(0, len(groups), per32)]
        for gset, gen, real, kpre in ((groups, g, "double", "k_sa"), (groups32, g32, "float", "k_saf")):
            base = 0
            tab = "a.boysf" if real == "float" else "a.boys"
            for r, gr in enumerate(gset):
                fname = f"acc_{g.tag}{'_f32' if real == 'float' else ''}_r{r}"
                code, _ = gen.emit_acc_role(fname, gr)
                funcs.append(code)
                kern.append(f"""
__device__ __forceinline__ void {kpre}_{g.tag}_r{r}_body(const StagedArgs& a) {{
    const {real}* __restrict__ sboys = {tab} + (size_t){g.L} * BOYS_BLK;  // Boys table of order L, through L1
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= staged_count(a)) return;
    const uint2 q = staged_quartet(a, t);
    const GPair bra = a.bra[q.x];
    const GPair ket = a.ket[q.y];
    {fname}(bra, ket, a.prims, sboys, reinterpret_cast<{real}*>(a.acc) + tcol(t, {len(keyidx)}) + {base} * TQ, TQ);
}}
__global__ void __launch_bounds__(RB_THREADS, 2 * RB_SCALE) {kpre}_{g.tag}_r{r}(StagedArgs a) {{ {kpre}_{g.tag}_r{r}_body(a); }}""")
                base += len(gr)
        og = prm["out_group3"]
        outroles = [list(range(i, min(i + og, g.nout))) for i in range(0, g.nout, og)]
        for r, outs in enumerate(outroles):
            code, _ = g.emit_hrr_role(f"hrr_{g.tag}_r{r}", outs, keyidx)
            code32, _ = g32.emit_hrr_role(f"hrr_{g.tag}_f32_r{r}", outs, keyidx)
            funcs += [code, code32]
            for kname, fname, real in ((f"k_sb_{g.tag}_r{r}", f"hrr_{g.tag}_r{r}", "double"),
                                       (f"k_sbf_{g.tag}_r{r}", f"hrr_{g.tag}_f32_r{r}", "float")):
                kern.append(f"""
__device__ __forceinline__ void {kname}_body(const StagedArgs& a) {{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= staged_count(a)) return;
    const uint2 q = staged_quartet(a, t);
    const GPair bra = a.bra[q.x];
    const GPair ket = a.ket[q.y];
    a.mx[tcol(t, {len(outroles)}) + {r} * TQ] =
        {fname}(bra, ket, reinterpret_cast<const {real}*>(a.acc) + tcol(t, {len(keyidx)}),
                reinterpret_cast<{real}*>(a.out) + tcol(t, {g.nout}) + {outs[0]} * TQ, TQ);
}}
__global__ void __launch_bounds__(RB_THREADS, RB_SCALE) {kname}(StagedArgs a) {{ {kname}_body(a); }}""")
        kern.append(merged_kernel(f"k_sam_{g.tag}", [f"k_sa_{g.tag}_r{r}" for r in range(len(groups))]))
        kern.append(merged_kernel(f"k_samf_{g.tag}", [f"k_saf_{g.tag}_r{r}" for r in range(len(groups32))]))
        kern.append(merged_kernel(f"k_sbm_{g.tag}", [f"k_sb_{g.tag}_r{r}" for r in range(len(outroles))], minb=1))
        kern.append(merged_kernel(f"k_sbmf_{g.tag}", [f"k_sbf_{g.tag}_r{r}" for r in range(len(outroles))], minb=1))
        reg.append(f"    k->ma64 = k_sam_{g.tag};\n    k->ma32 = k_samf_{g.tag};\n"
                   f"    k->mb64 = k_sbm_{g.tag};\n    k->mb32 = k_sbmf_{g.tag};")
        reg.append(f"    k->mode = 2;\n    k->nacc = {len(keyidx)};\n    k->nrole_a = {len(groups)};\n"
                   f"    k->nrole_a32 = {len(groups32)};\n"
                   f"    k->nrole_b = {len(outroles)};\n    k->nrole_b32 = {len(outroles)};")
        for r in range(len(groups)):
            reg.append(f"    k->sa64[{r}] = k_sa_{g.tag}_r{r};")
        for r in range(len(groups32)):
            reg.append(f"    k->sa32[{r}] = k_saf_{g.tag}_r{r};")
        for r in range(len(outroles)):
            reg.append(f"    k->sb64[{r}] = k_sb_{g.tag}_r{r};\n    k->sb32[{r}] = k_sbf_{g.tag}_r{r};")
        reg.append(f"    k->scat = k_scatter_staged<{NA}, {NB}, {NC}, {ND}>;\n"
                   f"    k->scat_smem = scat_smem_bytes({NA}, {NB}, {NC}, {ND});\n"
                   f"    k->scat32 = k_scatter_staged<{NA}, {NB}, {NC}, {ND}, float>;\n"
                   f"    k->scat32_smem = scat_smem_bytes({NA}, {NB}, {NC}, {ND}, 4);")
        reg.append(grouped_scatter_reg(NA, NB, NC, ND, prm))
        if bi == ki:
            reg.append(f"    k->diag0 = nullptr;\n    k->diag1 = nullptr;")
            reg.append(f"    k->dscat0 = k_scatter_diag<{NA}, {NB}, 0>;\n    k->dscat1 = k_scatter_diag<{NA}, {NB}, 1>;")
        info.update(roles=len(outroles), role_sizes=[len(x) for x in outroles], role_outs=outroles,
                    acc_groups=[[[list(k[2]), list(k[3]), k[0], k[1]] for k in gr] for gr in groups],
                    acc_groups32=[[[list(k[2]), list(k[3]), k[0], k[1]] for k in gr] for gr in groups32])
        assert len(groups) <= MAXR and len(outroles) <= MAXR
    if mode == "staged2":
        assert len(roles) <= MAXR
    info["mode"] = mode
    info["dims"] = [NA, NB, NC, ND]
    if bi != ki:
        reg.append("    k->diag0 = nullptr;\n    k->diag1 = nullptr;")
    if not (bi == ki and mode != "direct"):
        reg.append("    k->dscat0 = nullptr;\n    k->dscat1 = nullptr;")
    traits = f"HF_CLASS_TRAITS({ci}, {bi}, {ki}, {g.tag}, {g.nout}, {g.L})\n" if mode == "direct" else ""
    cuh = CLASS_CUH.format(A=g.A, B=g.B, C=g.C, D=g.D, roles=mode, body="\n\n".join(funcs))
    cu = CLASS_TU.format(A=g.A, B=g.B, C=g.C, D=g.D, kernels="\n".join(kern), ci=ci, bi=bi, ki=ki, tag=g.tag,
                         hdr=f"cls_{ci:02d}_{g.tag}.cuh", nout=g.nout, L=g.L, reg="\n".join(reg) + "\n",
                         roles=mode, traits=traits)
    return cuh, cu, info


CLASS_CUH = """// GENERATED by gen_eri.py -- do not edit.
// Device functions of quartet class ({A}{B}|{C}{D}): {roles} role(s).
#pragma once
#include "../types.cuh"

namespace hfgpu {{
{body}
}}  // namespace hfgpu
"""

CLASS_TU = """// GENERATED by gen_eri.py -- do not edit.
// Kernels of quartet class ({A}{B}|{C}{D}): {roles} role(s).
#include "../common.cuh"
#include "{hdr}"

namespace hfgpu {{
{kernels}
{traits}
void register_class_{ci}(ClassKernels* k) {{
{reg}    k->bi = {bi};
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
        cuh, cu, info = class_source(ci, bi, ki)
        flops[ci] = info
        base = os.path.join(outdir, f"cls_{ci:02d}_{info['tag']}")
        for ext, text in ((".cuh", cuh), (".cu", cu)):
            if not os.path.exists(base + ext) or open(base + ext).read() != text:
                with open(base + ext, "w") as fh:
                    fh.write(text)
        names.append(base + ".cu")
    # host dispatch used by the host-compiled check of the generated code
    lines = ["// GENERATED by gen_eri.py -- host dispatch of the class functions (tests only).", ""]
    for ci, info in flops.items():
        tag = info["tag"]
        nout = info["nout"]
        lines.append(f"inline void host_eri_{ci}(const GPair& b, const GPair& k, const PrimSoA& p, const double* t,")
        lines.append(f"                          const float* tf, double* out, int f32) {{")
        if info["mode"] == "direct":
            lines.append(f"    if (f32) {{ float o[{nout}]; eri_{tag}_f32(b, k, p, tf, o);")
            lines.append(f"        for (int i = 0; i < {nout}; ++i) out[i] = o[i]; }}")
            lines.append(f"    else eri_{tag}(b, k, p, t, out);")
        elif info["mode"] == "staged2":
            for r, outs in enumerate(info["role_outs"]):
                n = len(outs)
                idx = ", ".join(map(str, outs))
                lines.append(f"    if (!f32) {{ static const int ix[{n}] = {{{idx}}}; double o[{n}];")
                lines.append(f"      eri_{tag}_r{r}(b, k, p, t, o);")
                lines.append(f"      for (int i = 0; i < {n}; ++i) out[ix[i]] = o[i]; }}")
            for r, outs in enumerate(info["role_outs32"]):
                n = len(outs)
                idx = ", ".join(map(str, outs))
                lines.append(f"    if (f32) {{ static const int ix[{n}] = {{{idx}}}; float of[{n}];")
                lines.append(f"      eri_{tag}_f32_r{r}(b, k, p, tf, of);")
                lines.append(f"      for (int i = 0; i < {n}; ++i) out[ix[i]] = of[i]; }}")
        else:
            nacc = sum(len(g) for g in info["acc_groups"])
            lines.append(f"    static double acc[{nacc}];")
            lines.append(f"    static float accf[{nacc}];")
            base = 0
            for r, gr in enumerate(info["acc_groups"]):
                lines.append(f"    if (!f32) acc_{tag}_r{r}(b, k, p, t, acc + {base}, 1);")
                base += len(gr)
            base = 0
            for r, gr in enumerate(info["acc_groups32"]):
                lines.append(f"    if (f32) acc_{tag}_f32_r{r}(b, k, p, tf, accf + {base}, 1);")
                base += len(gr)
            for r, outs in enumerate(info["role_outs"]):
                n = len(outs)
                lines.append(f"    if (f32) {{ float of[{n}]; hrr_{tag}_f32_r{r}(b, k, accf, of, 1);")
                lines.append(f"      for (int i = 0; i < {n}; ++i) out[{outs[0]} + i] = of[i]; }}")
                lines.append(f"    else hrr_{tag}_r{r}(b, k, acc, out + {outs[0]}, 1);")
        lines.append("}")
        # the J/K scatter of a full block with stride 1
        na, nb_, nc, nd = info["dims"]
        lines.append(f"inline int host_scatter_{ci}(const double* e, double s, const GPair& b, const GPair& k,")
        lines.append(f"                             const double* P, double* G, int nb, bool jonly) {{")
        lines.append(f"    scatter_strided<{na}, {nb_}, {nc}, {nd}>(e, 1, s, b, k, P, G, nb, jonly);")
        lines.append("    return 0;")
        lines.append("}")
    lines.append("typedef void (*HostEri)(const GPair&, const GPair&, const PrimSoA&, const double*, const float*, double*, int);")
    lines.append("typedef int (*HostScat)(const double*, double, const GPair&, const GPair&, const double*, double*, int, bool);")
    lines.append("static const HostEri HOST_ERI[] = {" + ", ".join(f"host_eri_{ci}" for ci in flops) + "};")
    lines.append("static const HostScat HOST_SCAT[] = {" + ", ".join(f"host_scatter_{ci}" for ci in flops) + "};")
    txt = "\n".join(lines) + "\n"
    inc = '#include "../scatter.cuh"\n'
    inc += "".join(f'#include "cls_{ci:02d}_{info["tag"]}.cuh"\n' for ci, info in flops.items())
    inc += "namespace hfgpu {\n#include \"host_dispatch.inc\"\n}\n"
    cl = class_list()
    tab = ["// GENERATED by gen_eri.py -- quartet classes over the GPU pair types.",
           f"#define HF_NPT {len(PAIR_TYPES)}",
           f"#define HF_NCLS {len(cl)}",
           "#define HF_CLASS_BI_LIST " + ", ".join(str(b) for b, _ in cl),
           "#define HF_CLASS_KI_LIST " + ", ".join(str(k) for _, k in cl),
           "#define HF_FOR_EACH_CLASS(X) " + " ".join(f"X({c})" for c in range(len(cl))),
           "#define HF_PAIR_NAMES " + ", ".join(f'"{a}{b}"' for a, b in PAIR_TYPES), ""]
    ct = os.path.join(outdir, "class_table.inc")
    if not os.path.exists(ct) or open(ct).read() != "\n".join(tab):
        with open(ct, "w") as fh:
            fh.write("\n".join(tab))
    ai = os.path.join(outdir, "all_classes.inc")
    if not os.path.exists(ai) or open(ai).read() != inc:
        with open(ai, "w") as fh:
            fh.write(inc)
    hd = os.path.join(outdir, "host_dispatch.inc")
    if not os.path.exists(hd) or open(hd).read() != txt:
        with open(hd, "w") as fh:
            fh.write(txt)
    import json
    fl = os.path.join(outdir, "class_flops.json")
    txt = json.dumps(flops, indent=1)
    if not os.path.exists(fl) or open(fl).read() != txt:
        with open(fl, "w") as fh:
            fh.write(txt)
    return names


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)), "generated"))
