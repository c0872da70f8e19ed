// Host-side set-up of the B200 Fock builder (no CUDA): shell-pair lists in
// the reference's enumeration order, primitive-pair data with the negab
// screen (precalc_kabs.f90:38-295) and the Boys Taylor table.  Shared by the
// library and by the host-compiled check of the generated class code.
#pragma once
#include <cmath>
#include <vector>

#include "../../include/hfgpu_basis.h"
#include "types.cuh"

namespace hfgpu {

struct HostPair {
    GPair g;
    int refcls;   // reference class index 0..9 (ss sp sd sl pp pd pl dd dl ll)
    int refpos;   // position in the reference's class list
};

inline int ref_rank(int t) { return t == HFGPU_SHELL_S ? 0 : t == HFGPU_SHELL_P ? 1 : t == HFGPU_SHELL_D ? 2 : 3; }
inline int nfunc_of(int t) { return t == HFGPU_SHELL_S ? 1 : t == HFGPU_SHELL_P ? 3 : t == HFGPU_SHELL_D ? 5 : 4; }

// reference class (ss sp sd sl pp pd pl dd dl ll) of a rank pair (r1 <= r2)
inline int ref_class(int r1, int r2) {
    static const int tab[4][4] = {{0, 1, 2, 3}, {-1, 4, 5, 6}, {-1, -1, 7, 8}, {-1, -1, -1, 9}};
    return tab[r1][r2];
}
// GPU pair type of a reference class, and whether the GPU pair swaps the
// reference's (first, second) order (the GPU puts the larger shell first).
inline int gpu_type_of_ref(int rc, bool* swap) {
    switch (rc) {
        case 0: *swap = false; return 0;  // ss -> SS
        case 3: *swap = true; return 1;   // sl -> LS
        case 9: *swap = false; return 2;  // ll -> LL
        case 2: *swap = true; return 3;   // sd -> DS
        case 8: *swap = false; return 4;  // dl -> DL
        case 7: *swap = false; return 5;  // dd -> DD
        case 1: *swap = true; return 6;   // sp -> PS
        case 6: *swap = true; return 7;   // pl -> LP
        case 4: *swap = false; return 8;  // pp -> PP
        case 5: *swap = true; return 9;   // pd -> DP
        default: *swap = false; return -1;
    }
}
constexpr int GPU_TO_REF[NPT] = {0, 3, 9, 2, 8, 7, 1, 6, 4, 5};

// One shell pair in GPU orientation with its surviving primitive pairs
// appended to prims: K_ab = sqrt(2 pi^2.5) exp(-ab/p r^2)/p d_a d_b, dropped
// when |K_ab|/sqrt(p) < 1e-12 (precalc_kabs.f90:103-110).
inline GPair make_pair(const hfgpu_basis* B, int a, int b, std::vector<GPrim>& prims) {
    const double PI = 3.141592653589793238462643383279502884197;
    const double RT2PI54 = std::sqrt(2.0 * PI * PI * std::sqrt(PI));
    const int MP = B->maxprim;
    GPair g;
    for (int x = 0; x < 3; ++x) {
        g.A[x] = B->xsh[3 * a + x];
        g.B[x] = B->xsh[3 * b + x];
    }
    g.sa = a;
    g.sb = b;
    g.aoa = B->aosh[a];
    g.aob = B->aosh[b];
    g.p0 = (int)prims.size();
    g.ps = 1;
    g.pad = 0;
    double r2ab = 0;
    for (int x = 0; x < 3; ++x) r2ab += (g.A[x] - g.B[x]) * (g.A[x] - g.B[x]);
    for (int za = 0; za < B->nzet[a]; ++za)
        for (int zb = 0; zb < B->nzet[b]; ++zb) {
            double ea = B->zeta[(size_t)a * MP + za], eb = B->zeta[(size_t)b * MP + zb];
            double p = ea + eb, pm1 = 1.0 / p, q = ea * eb * pm1;
            double K = RT2PI54 * std::exp(-q * r2ab) * pm1 * B->djk[(size_t)a * MP + za] * B->djk[(size_t)b * MP + zb];
            if (std::fabs(K) * std::sqrt(pm1) < 1e-12) continue;  // negab
            GPrim gp;
            gp.p = p;
            for (int x = 0; x < 3; ++x) gp.P[x] = (ea * g.A[x] + eb * g.B[x]) * pm1;
            gp.K = K;
            gp.w1 = B->shtyp[a] == HFGPU_SHELL_L ? B->djkl[(size_t)a * MP + za] : 1.0;
            gp.w2 = B->shtyp[b] == HFGPU_SHELL_L ? B->djkl[(size_t)b * MP + zb] : 1.0;
            gp.pad = 0.0;
            prims.push_back(gp);
        }
    g.np = (int)prims.size() - g.p0;
    return g;
}

// Pair lists per GPU pair type, in the reference's enumeration order
// (precalc_kabs.f90:38-90); returns the number of pairs.
inline int build_pairs(const hfgpu_basis* B, std::vector<HostPair>* pairs, std::vector<GPrim>& prims,
                       std::vector<int>& refcount) {
    refcount.assign(10, 0);
    int n = 0;
    for (int s1 = 0; s1 < B->nsh; ++s1)
        for (int s2 = 0; s2 <= s1; ++s2) {
            int r1 = s1, r2 = s2;
            if (ref_rank(B->shtyp[r1]) > ref_rank(B->shtyp[r2])) std::swap(r1, r2);
            int rc = ref_class(ref_rank(B->shtyp[r1]), ref_rank(B->shtyp[r2]));
            bool swp = false;
            int gt = gpu_type_of_ref(rc, &swp);
            HostPair hp;
            hp.refcls = rc;
            hp.refpos = refcount[rc]++;
            hp.g = make_pair(B, swp ? r2 : r1, swp ? r1 : r2, prims);
            pairs[gt].push_back(hp);
            ++n;
        }
    return n;
}

inline long double boys_series(int m, long double T) {
    // F_m(T) = e^-T sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1))
    long double term = 1.0L / (2 * m + 1), sum = term;
    for (int k = 1; k < 400; ++k) {
        term *= 2.0L * T / (2 * m + 2 * k + 1);
        sum += term;
        if (term < sum * 1e-22L) break;
    }
    return expl(-T) * sum;
}

// Boys Taylor tables: c_k = F_{M+k}(T_j) (-1)^k / k!, M = 0..8, T_j = j/8;
// each order's block ends with exp(-T_j) for the downward recursion.
inline void build_boys_table(std::vector<double>& bt, std::vector<float>& btf) {
    bt.assign((size_t)(BOYS_MMAX + 1) * BOYS_BLK, 0.0);
    btf.assign(bt.size(), 0.0f);
    for (int M = 0; M <= BOYS_MMAX; ++M)
        for (int j = 0; j < BOYS_NPT; ++j) {
            long double T = j / 8.0L, fact = 1.0L;
            for (int k = 0; k < BOYS_K; ++k) {
                if (k) fact *= k;
                long double v = boys_series(M + k, T) / fact * ((k & 1) ? -1.0L : 1.0L);
                size_t i = (size_t)M * BOYS_BLK + (size_t)j * BOYS_K + k;
                bt[i] = (double)v;
                btf[i] = (float)v;
            }
            const size_t ie = (size_t)M * BOYS_BLK + (size_t)BOYS_NPT * BOYS_K + j;
            bt[ie] = (double)expl(-T);
            btf[ie] = (float)expl(-T);
        }
}

// Structure-of-arrays copy of primitive pairs: 8 arrays of n doubles
// (p, Px, Py, Pz, K, w1, w2, 1/(2p)) back to back.
inline std::vector<double> prims_soa(const std::vector<GPrim>& prims) {
    // four arrays of (field, field) pairs, 2n doubles each (see PrimSoA)
    const size_t n = prims.size();
    std::vector<double> s(8 * n);
    for (size_t i = 0; i < n; ++i) {
        s[2 * i] = prims[i].p;
        s[2 * i + 1] = prims[i].P[0];
        s[2 * n + 2 * i] = prims[i].P[1];
        s[2 * n + 2 * i + 1] = prims[i].P[2];
        s[4 * n + 2 * i] = prims[i].K;
        s[4 * n + 2 * i + 1] = prims[i].w1;
        s[6 * n + 2 * i] = prims[i].w2;
        s[6 * n + 2 * i + 1] = 0.5 / prims[i].p;
    }
    return s;
}
inline PrimSoA soa_view(const double* base, size_t n) {
    const PrimVec* v = reinterpret_cast<const PrimVec*>(base);
    return PrimSoA{v, v + n, v + 2 * n, v + 3 * n};
}

}  // namespace hfgpu
