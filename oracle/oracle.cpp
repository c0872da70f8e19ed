/*
 * CPU oracle for the direct-SCF Fock build -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is a CPU restatement of the reference (brichjnh/hfcode, Fortran)
 * hot path.  It exists to check the CUDA product: only the tests, the smoke
 * check and the CPU-baseline leg of bench.py load it.  The product library
 * never links or calls it.
 *
 * Parity is UNPINNED by the reference itself: the reference ships no tests,
 * golden vectors or outputs, and it cannot be compiled here (Fortran, no
 * Fortran compiler).  The restatement is pinned instead by known-answer
 * checks in tests/ (Boys function against arbitrary precision, ERIs against
 * an independent McMurchie-Davidson implementation, J/K against a brute-force
 * contraction of the full ERI tensor).
 *
 * What is restated, with the reference lines it follows:
 *   Boys function, 4 regimes incl. the 1e-3 cubic-Taylor grid
 *       boys.f90:7-158, index_functions.f90:171-226
 *   primitive-pair data and the negab primitive screen (|K_ab|/sqrt(p)<1e-12)
 *       precalc_kabs.f90:13-20,94-295
 *   shell-pair class lists (ss,sp,sd,sl,pp,pd,pl,dd,dl,ll) and their order
 *       precalc_kabs.f90:38-90
 *   contracted ERIs: Obara-Saika recursion on all four centres with the
 *       L-shell p/s ratio weights and the Cartesian->spherical d transform
 *       s_sp_l_terms.f90, s_p_d_terms.f90, s_d_l_terms.f90 (e.g. llll at
 *       s_d_l_terms.f90:1786-1905), index_functions.f90:147-168; the Boys
 *       routine is picked by total angular momentum as each i2e_* does
 *   evaluate_maxdm incl. its d-l block (rows d0..d3, columns l0..l3 plus the
 *       function after the l shell)              evaluate_maxdm.f90:82-89
 *   Schwarz factors, descending sort and the inclusive find_threshold cut
 *       fock_build_initial_diag.f90:31-53,...,684-811; index_sort.f90:95-119
 *   fock_build_initial_diag   element skip |e|>intthresh, no density screen
 *   fock_build_diag           schw^2*max(D_ab,D_aa/4,D_bb/4) < thr skip
 *                             (fock_build_diag.f90:17-36)
 *   fock_build_non_diag       schw_ab*schw_cd*max(Dcoul,Dexch/4) < thr skip,
 *                             post-skip max|e| < thr (fock_build_non_diag.f90:52-117)
 *   fock_build_non_diag_j_only  Coulomb only (fock_build_non_diag_j.f90:50-90)
 *
 * Scatter: the reference's per-case branches all add the standard RHF
 * F += J(P) - K(P)/2 contribution of each unique AO quartet to both
 * triangles.  Here every ordered component of a shell quartet is visited with
 * the quartet's uniform degeneracy weight s (1/8 x the product of the bra,
 * ket and bra-ket permutation counts), accumulated into one triangle-agnostic
 * buffer G, and F += G + G^T at the end -- the same sums, in another order.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <numeric>
#include <tuple>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/hfgpu_basis.h"

namespace {

const double PI = 3.141592653589793238462643383279502884197;
const double TWOPI5 = 2.0 * PI * PI * std::sqrt(PI);
const double RT2PI54 = std::sqrt(TWOPI5);
const double INTTHRESH = 1e-10;      // molprops.f90:162
const double SHTHRESH = 1e-11;       // molprops.f90:163
const double EXTRATHRESH = 1e-12;    // precalc_kabs.f90:13
const int MAXGAMMA = 50, MAXBOYS = 9, NGAMMA = 10000;
const double TWODELTA = 1e-3;

/* ---------------- Boys function (boys.f90, index_functions.f90) -------- */
struct BoysTables {
    double gammrats[MAXGAMMA + 1][MAXBOYS + 4];
    std::vector<double> vals;  // [i][j][c] = boysfuncvals(c, j, i)
    double zeroarg[MAXBOYS + 1], lrfac[MAXBOYS + 1], mrfac[MAXBOYS + 1];
    BoysTables() {
        for (int i = 0; i <= MAXGAMMA; ++i)
            for (int j = 0; j <= MAXBOYS + 3; ++j)
                gammrats[i][j] = std::tgamma(j + 0.5) / std::tgamma(i + j + 1.5);
        for (int i = 0; i <= MAXBOYS; ++i) zeroarg[i] = 1.0 / (1 + 2 * i);
        for (int i = 1; i <= MAXBOYS; ++i) {
            lrfac[i] = i - 0.5;
            mrfac[i] = 2.0 / (2 * (i - 1) + 1);
        }
        vals.resize((size_t)(NGAMMA + 1) * (MAXBOYS + 1) * 4);
        for (int i = 0; i <= NGAMMA; ++i) {
            double x = (i + 0.5) * TWODELTA;
            double bf[MAXBOYS + 4] = {0};
            double xpow = 1.0, efac = std::exp(-x) / 2.0;
            for (int jn = 0; jn <= MAXGAMMA; ++jn) {
                for (int j = 0; j <= MAXBOYS + 3; ++j) bf[j] += xpow * gammrats[jn][j];
                xpow *= x;
            }
            for (int j = 0; j <= MAXBOYS + 3; ++j) bf[j] *= efac;
            for (int j = 0; j <= MAXBOYS; ++j) {
                double* v = &vals[((size_t)i * (MAXBOYS + 1) + j) * 4];
                v[0] = bf[j] + x * bf[j + 1] + .5 * x * x * bf[j + 2] + x * x * x * bf[j + 3] / 6.0;
                v[1] = bf[j + 1] + x * bf[j + 2] + .5 * x * x * bf[j + 3];
                v[2] = .5 * bf[j + 2] + .5 * x * bf[j + 3];
                v[3] = bf[j + 3] / 6.0;
            }
        }
    }
    inline double taylor(int j, int m, double x) const {
        const double* v = &vals[((size_t)j * (MAXBOYS + 1) + m) * 4];
        return v[0] - x * (v[1] - x * (v[2] - x * v[3]));
    }
};

const BoysTables& boys_tables() {
    static BoysTables t;
    return t;
}

const double HSQRTPI = std::sqrt(PI) / 2.0;

// boys_0 / boys_1 / boys_2 / boys_n dispatched by the highest order n, as
// each i2e_* kernel calls the routine for its total angular momentum.
void boys(int n, double x, double* fn) {
    const BoysTables& T = boys_tables();
    const double vsmall = 1e-15, lr = 28.0;
    if (n == 0) {
        if (x < vsmall) { fn[0] = 1.0; return; }
        if (x > lr) { fn[0] = HSQRTPI / std::sqrt(x); return; }
        if (x >= 2.0 && x <= lr) { double s = std::sqrt(x); fn[0] = HSQRTPI * std::erf(s) / s; return; }
        int j = (int)(x / TWODELTA);
        fn[0] = T.taylor(j, 0, x);
        return;
    }
    if (n == 1) {
        if (x < vsmall) { fn[0] = T.zeroarg[0]; fn[1] = T.zeroarg[1]; return; }
        if (x > lr) { fn[0] = HSQRTPI / std::sqrt(x); fn[1] = fn[0] * .5 / x; return; }
        if (x >= 4.0 && x <= lr) {
            double s = std::sqrt(x);
            fn[0] = HSQRTPI * std::erf(s) / s;
            fn[1] = (fn[0] - std::exp(-x)) / (2.0 * x);
            return;
        }
        int j = (int)(x / TWODELTA);
        fn[0] = T.taylor(j, 0, x); fn[1] = T.taylor(j, 1, x);
        return;
    }
    if (n == 2) {
        if (x < vsmall) { for (int i = 0; i <= 2; ++i) fn[i] = T.zeroarg[i]; return; }
        if (x > lr) {
            fn[0] = HSQRTPI / std::sqrt(x); fn[1] = fn[0] * .5 / x; fn[2] = fn[1] * 1.5 / x;
            return;
        }
        if (x >= 8.0 && x <= lr) {
            double s = std::sqrt(x);
            fn[0] = HSQRTPI * std::erf(s) / s;
            double efac = .5 * std::exp(-x);
            fn[1] = (.5 * fn[0] - efac) / x;
            fn[2] = (1.5 * fn[1] - efac) / x;
            return;
        }
        int j = (int)(x / TWODELTA);
        double efac = .5 * std::exp(-x);
        fn[2] = T.taylor(j, 2, x);
        fn[1] = (x * fn[2] + efac) * 2.0 / 3.0;
        fn[0] = (x * fn[1] + efac) * 2.0;
        return;
    }
    if (x < vsmall) { for (int i = 0; i <= n; ++i) fn[i] = T.zeroarg[i]; return; }
    if (x > lr) {
        fn[0] = HSQRTPI / std::sqrt(x);
        for (int i = 1; i <= n; ++i) fn[i] = fn[i - 1] * T.lrfac[i] / x;
        return;
    }
    if (x >= 8.0 && x <= lr) {
        double s = std::sqrt(x);
        fn[0] = HSQRTPI * std::erf(s) / s;
        double efac = .5 * std::exp(-x);
        for (int i = 0; i < n; ++i) fn[i + 1] = (T.lrfac[i + 1] * fn[i] - efac) / x;
        return;
    }
    int j = (int)(x / TWODELTA);
    double efac = .5 * std::exp(-x);
    fn[n] = T.taylor(j, n, x);
    for (int i = n; i >= 1; --i) fn[i - 1] = (x * fn[i] + efac) * T.mrfac[i];
}

/* ---------------- Cartesian components ------------------------------- */
struct Cart { int8_t x, y, z; };
// indexps order (index_functions.f90:54-66): l=1: x,y,z; l=2: xx,xy,xz,yy,yz,zz
const Cart CART_S[1] = {{0, 0, 0}};
const Cart CART_P[3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
const Cart CART_L[4] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
const Cart CART_D[6] = {{2, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 2, 0}, {0, 1, 1}, {0, 0, 2}};

int ncart(int t) { return t == HFGPU_SHELL_S ? 1 : t == HFGPU_SHELL_P ? 3 : t == HFGPU_SHELL_L ? 4 : 6; }
int nfunc(int t) { return t == HFGPU_SHELL_S ? 1 : t == HFGPU_SHELL_P ? 3 : t == HFGPU_SHELL_L ? 4 : 5; }
int lmax(int t) { return t == HFGPU_SHELL_S ? 0 : t == HFGPU_SHELL_D ? 2 : 1; }
const Cart* carts(int t) {
    return t == HFGPU_SHELL_S ? CART_S : t == HFGPU_SHELL_P ? CART_P : t == HFGPU_SHELL_L ? CART_L : CART_D;
}

// matharmond (index_functions.f90:158-167): spherical d (z2,xz,yz,xy,x2-y2)
// from Cartesian (xx,xy,xz,yy,yz,zz)
double harm(int s, int c) {
    struct Tab {
        double M[5][6];
        Tab() {
            std::memset(M, 0, sizeof(M));
            M[0][5] = 1.0; M[0][0] = -.5; M[0][3] = -.5;
            M[1][2] = std::sqrt(3.0);
            M[2][4] = std::sqrt(3.0);
            M[3][1] = std::sqrt(3.0);
            M[4][0] = std::sqrt(3.0) / 2.0; M[4][3] = -std::sqrt(3.0) / 2.0;
        }
    };
    static const Tab tab;  // initialised once, thread-safe
    return tab.M[s][c];
}

/* ---------------- 4-centre Obara-Saika plan ---------------------------- */
// Coefficient slots computed once per primitive quartet.
enum { C_PA = 0, C_PB = 3, C_QC = 6, C_QD = 9, C_WP = 12, C_WQ = 15,
       C_H2P = 18, C_RH2P = 19, C_H2Q = 20, C_RH2Q = 21, C_H2PQ = 22, C_NCOEF = 23 };

struct Term { int16_t coef; int16_t mult; int32_t child; };
struct Op { int m; int nterm; int first; };  // nterm==0 -> base [00|00]^m

struct Plan {
    int maxm = 0;
    std::vector<Op> ops;
    std::vector<Term> terms;
    std::vector<int> target;  // op index per cartesian (a,b,c,d) target
    std::vector<uint8_t> wpat;  // per target: bit c set when centre c's component is an L-shell p
};

struct Key {
    int8_t e[12]; int8_t m;
    bool operator<(const Key& o) const {
        int c = std::memcmp(e, o.e, 12);
        if (c) return c < 0;
        return m < o.m;
    }
};

struct PlanBuilder {
    Plan plan;
    std::map<Key, int> idx;
    int get(const Key& k) {
        auto it = idx.find(k);
        if (it != idx.end()) return it->second;
        // pick the first centre with angular momentum, then its first axis
        int ctr = -1, ax = -1;
        for (int c = 0; c < 4 && ctr < 0; ++c)
            for (int a = 0; a < 3; ++a)
                if (k.e[3 * c + a] > 0) { ctr = c; ax = a; break; }
        Op op; op.m = k.m; op.nterm = 0; op.first = 0;
        std::vector<Term> tl;
        if (ctr >= 0) {
            Key r = k; r.e[3 * ctr + ax] -= 1;
            auto add = [&](int coef, int mult, Key kk) {
                for (int q = 0; q < 12; ++q) if (kk.e[q] < 0) return;
                if (mult == 0) return;
                int ch = get(kk);
                tl.push_back(Term{(int16_t)coef, (int16_t)mult, ch});
            };
            bool bra = ctr < 2;
            int cgeo = ctr == 0 ? C_PA : ctr == 1 ? C_PB : ctr == 2 ? C_QC : C_QD;
            int cw = bra ? C_WP : C_WQ;
            Key r1 = r; r1.m = k.m + 1;
            add(cgeo + ax, 1, r);
            add(cw + ax, 1, r1);
            // same-electron terms
            int s0 = bra ? 0 : 2;
            for (int c = s0; c < s0 + 2; ++c) {
                int n = r.e[3 * c + ax];
                if (n <= 0) continue;
                Key t0 = r; t0.e[3 * c + ax] -= 1;
                Key t1 = t0; t1.m = k.m + 1;
                add(bra ? C_H2P : C_H2Q, n, t0);
                add(bra ? C_RH2P : C_RH2Q, n, t1);
            }
            // other-electron terms
            int o0 = bra ? 2 : 0;
            for (int c = o0; c < o0 + 2; ++c) {
                int n = r.e[3 * c + ax];
                if (n <= 0) continue;
                Key t1 = r; t1.e[3 * c + ax] -= 1; t1.m = k.m + 1;
                add(C_H2PQ, n, t1);
            }
        }
        op.first = (int)plan.terms.size();
        op.nterm = (int)tl.size();
        plan.terms.insert(plan.terms.end(), tl.begin(), tl.end());
        if (k.m > plan.maxm) plan.maxm = k.m;
        int id = (int)plan.ops.size();
        plan.ops.push_back(op);
        idx[k] = id;
        return id;
    }
};

/* ---------------- Oracle state ---------------------------------------- */
struct PrimPair { double p, Px, Py, Pz, K; int za, zb; };

struct PairData {
    int sh1, sh2;      // order as stored in the reference's class list
    std::vector<PrimPair> prims;  // non-negab primitive pairs only
};

// class order of the reference's pair lists: ss sp sd sl pp pd pl dd dl ll
enum { CSS = 0, CSP, CSD, CSL, CPP, CPD, CPL, CDD, CDL, CLL, NCLASS };

struct Oracle {
    int nsh, nb, maxprim;
    std::vector<int> shtyp, nzet, atsh, aosh;
    std::vector<double> xsh, zeta, djk, djkl;
    std::vector<std::vector<int>> cls;   // per class: pair ids (list order)
    std::vector<PairData> pairs;         // by pair id
    std::vector<int> pairid;             // nsh*nsh -> pair id
    std::vector<double> schw;            // by pair id
    std::vector<int> order[NCLASS];      // sorted list positions -> pair ids
    int last[NCLASS];
    bool have_schwarz = false;
    std::map<std::tuple<int, int, int, int>, Plan> plans;
    // statistics of the last build
    long long n_screen_pass = 0, n_scatter = 0;
    std::vector<long long> class_pass, class_scatter;  // 100 = 10x10 class pairs

    const Plan& plan_for(int t1, int t2, int t3, int t4) {
        auto key = std::make_tuple(t1, t2, t3, t4);
        auto it = plans.find(key);
        if (it != plans.end()) return it->second;
        PlanBuilder b;
        int n1 = ncart(t1), n2 = ncart(t2), n3 = ncart(t3), n4 = ncart(t4);
        const Cart *c1 = carts(t1), *c2 = carts(t2), *c3 = carts(t3), *c4 = carts(t4);
        for (int i = 0; i < n1; ++i) for (int j = 0; j < n2; ++j)
        for (int k = 0; k < n3; ++k) for (int l = 0; l < n4; ++l) {
            Key key4;
            const Cart* cs[4] = {&c1[i], &c2[j], &c3[k], &c4[l]};
            for (int c = 0; c < 4; ++c) {
                key4.e[3 * c] = cs[c]->x; key4.e[3 * c + 1] = cs[c]->y; key4.e[3 * c + 2] = cs[c]->z;
            }
            key4.m = 0;
            b.plan.target.push_back(b.get(key4));
            const int ts[4] = {t1, t2, t3, t4};
            uint8_t pat = 0;
            for (int c = 0; c < 4; ++c)
                if (ts[c] == HFGPU_SHELL_L && (cs[c]->x + cs[c]->y + cs[c]->z) == 1) pat |= (uint8_t)(1 << c);
            b.plan.wpat.push_back(pat);
        }
        const Plan& pl = plans.emplace(key, std::move(b.plan)).first->second;
        fast[tix(t1)][tix(t2)][tix(t3)][tix(t4)] = &pl;
        return pl;
    }

    // Plans by shell-type index (S P D L -> 0..3), filled by plan_for; the
    // OpenMP regions only read this table (init builds every plan they use).
    const Plan* fast[4][4][4][4] = {};
    static int tix(int t) { return t == HFGPU_SHELL_S ? 0 : t == HFGPU_SHELL_P ? 1 : t == HFGPU_SHELL_D ? 2 : 3; }
    const Plan& plan_fast(int t1, int t2, int t3, int t4) {
        const Plan* p = fast[tix(t1)][tix(t2)][tix(t3)][tix(t4)];
        return p ? *p : plan_for(t1, t2, t3, t4);
    }

    int classof(int ta, int tb) const {
        auto r = [](int t) { return t == HFGPU_SHELL_S ? 0 : t == HFGPU_SHELL_P ? 1 : t == HFGPU_SHELL_D ? 2 : 3; };
        int a = r(ta), b = r(tb);
        if (a > b) std::swap(a, b);
        static const int tab[4][4] = {{CSS, CSP, CSD, CSL}, {-1, CPP, CPD, CPL}, {-1, -1, CDD, CDL}, {-1, -1, -1, CLL}};
        return tab[a][b];
    }

    void init(const hfgpu_basis* B) {
        nsh = B->nsh; nb = B->nb; maxprim = B->maxprim;
        shtyp.assign(B->shtyp, B->shtyp + nsh);
        nzet.assign(B->nzet, B->nzet + nsh);
        atsh.assign(B->atsh, B->atsh + nsh);
        aosh.assign(B->aosh, B->aosh + nsh);
        xsh.assign(B->xsh, B->xsh + 3 * nsh);
        zeta.assign(B->zeta, B->zeta + (size_t)nsh * maxprim);
        djk.assign(B->djk, B->djk + (size_t)nsh * maxprim);
        djkl.assign(B->djkl, B->djkl + (size_t)nsh * maxprim);
        cls.assign(NCLASS, {});
        pairid.assign((size_t)nsh * nsh, -1);
        // precalc_kabs.f90:38-90: pair lists, lower-"rank" shell type first
        auto rank = [](int t) { return t == HFGPU_SHELL_S ? 0 : t == HFGPU_SHELL_P ? 1 : t == HFGPU_SHELL_D ? 2 : 3; };
        for (int s1 = 0; s1 < nsh; ++s1)
            for (int s2 = 0; s2 <= s1; ++s2) {
                int a = s1, b = s2;
                if (rank(shtyp[a]) > rank(shtyp[b])) std::swap(a, b);
                int c = classof(shtyp[a], shtyp[b]);
                PairData pd; pd.sh1 = a; pd.sh2 = b;
                double r2 = 0;
                for (int x = 0; x < 3; ++x) {
                    double d = xsh[3 * a + x] - xsh[3 * b + x];
                    r2 += d * d;
                }
                for (int za = 0; za < nzet[a]; ++za)
                    for (int zb = 0; zb < nzet[b]; ++zb) {
                        double ea = zeta[(size_t)a * maxprim + za], eb = zeta[(size_t)b * maxprim + zb];
                        double p = ea + eb, pm1 = 1.0 / p, q = ea * eb * pm1;
                        double dd = djk[(size_t)a * maxprim + za] * djk[(size_t)b * maxprim + zb];
                        double K = RT2PI54 * std::exp(-q * r2) * pm1 * dd;
                        if (std::fabs(K) * std::sqrt(pm1) < EXTRATHRESH) continue;  // negab
                        PrimPair pp;
                        pp.p = p; pp.K = K; pp.za = za; pp.zb = zb;
                        pp.Px = (ea * xsh[3 * a] + eb * xsh[3 * b]) * pm1;
                        pp.Py = (ea * xsh[3 * a + 1] + eb * xsh[3 * b + 1]) * pm1;
                        pp.Pz = (ea * xsh[3 * a + 2] + eb * xsh[3 * b + 2]) * pm1;
                        pd.prims.push_back(pp);
                    }
                int id = (int)pairs.size();
                pairs.push_back(pd);
                pairid[(size_t)s1 * nsh + s2] = id;
                pairid[(size_t)s2 * nsh + s1] = id;
                cls[c].push_back(id);
            }
        schw.assign(pairs.size(), 0.0);
        for (int c = 0; c < NCLASS; ++c) last[c] = 0;
        // build every class-pair recursion plan up front (the OpenMP
        // regions below only read the plan map)
        for (int ca = 0; ca < NCLASS; ++ca)
            for (int cb = 0; cb < NCLASS; ++cb) {
                if (cls[ca].empty() || cls[cb].empty()) continue;
                const PairData& A = pairs[cls[ca][0]];
                const PairData& C = pairs[cls[cb][0]];
                plan_for(shtyp[A.sh1], shtyp[A.sh2], shtyp[C.sh1], shtyp[C.sh2]);
            }
        class_pass.assign(NCLASS * NCLASS, 0);
        class_scatter.assign(NCLASS * NCLASS, 0);
    }

    // Contracted ERI block of (s1 s2|s3 s4) over the pairs' stored prims.
    // out[((i*n2+j)*n3+k)*n4+l] in each shell's function order.  The plan,
    // its per-target L-weight pattern and every work array are looked up or
    // reused, so a call allocates nothing once its thread has run one quartet.
    void eri(int pab, int pcd, double* out) {
        const PairData& A = pairs[pab];
        const PairData& C = pairs[pcd];
        int s[4] = {A.sh1, A.sh2, C.sh1, C.sh2};
        int t[4] = {shtyp[s[0]], shtyp[s[1]], shtyp[s[2]], shtyp[s[3]]};
        const Plan& pl = plan_fast(t[0], t[1], t[2], t[3]);
        int nc[4] = {ncart(t[0]), ncart(t[1]), ncart(t[2]), ncart(t[3])};
        int ncart4 = nc[0] * nc[1] * nc[2] * nc[3];
        int L = lmax(t[0]) + lmax(t[1]) + lmax(t[2]) + lmax(t[3]);
        thread_local std::vector<double> acc, v, cur, nx;
        acc.assign(ncart4, 0.0);
        if (v.size() < pl.ops.size()) v.resize(pl.ops.size());
        const double* X[4] = {&xsh[3 * s[0]], &xsh[3 * s[1]], &xsh[3 * s[2]], &xsh[3 * s[3]]};
        double fm[32];
        double cf[C_NCOEF];
        for (const PrimPair& pa : A.prims) {
            for (const PrimPair& pc : C.prims) {
                double p = pa.p, q = pc.p;
                double ooppq = 1.0 / (p + q);
                double rho = p * q * ooppq;
                double P[3] = {pa.Px, pa.Py, pa.Pz}, Q[3] = {pc.Px, pc.Py, pc.Pz};
                double rpq2 = 0;
                for (int x = 0; x < 3; ++x) rpq2 += (P[x] - Q[x]) * (P[x] - Q[x]);
                boys(L, rho * rpq2, fm);
                double pref = pa.K * pc.K * std::sqrt(ooppq);
                for (int x = 0; x < 3; ++x) {
                    double W = (p * P[x] + q * Q[x]) * ooppq;
                    cf[C_PA + x] = P[x] - X[0][x];
                    cf[C_PB + x] = P[x] - X[1][x];
                    cf[C_QC + x] = Q[x] - X[2][x];
                    cf[C_QD + x] = Q[x] - X[3][x];
                    cf[C_WP + x] = W - P[x];
                    cf[C_WQ + x] = W - Q[x];
                }
                cf[C_H2P] = 0.5 / p;
                cf[C_RH2P] = -0.5 / p * (rho / p);
                cf[C_H2Q] = 0.5 / q;
                cf[C_RH2Q] = -0.5 / q * (rho / q);
                cf[C_H2PQ] = 0.5 * ooppq;
                const size_t nops = pl.ops.size();
                for (size_t o = 0; o < nops; ++o) {
                    const Op& op = pl.ops[o];
                    if (op.nterm == 0) { v[o] = pref * fm[op.m]; continue; }
                    double sum = 0;
                    const Term* tm = &pl.terms[op.first];
                    for (int tt = 0; tt < op.nterm; ++tt) sum += cf[tm[tt].coef] * tm[tt].mult * v[tm[tt].child];
                    v[o] = sum;
                }
                // weights of L-shell p components (s_d_l_terms.f90:1885-1896):
                // wt[pattern] for the 16 patterns of p-component centres
                double w[4];
                w[0] = djkl[(size_t)s[0] * maxprim + pa.za];
                w[1] = djkl[(size_t)s[1] * maxprim + pa.zb];
                w[2] = djkl[(size_t)s[2] * maxprim + pc.za];
                w[3] = djkl[(size_t)s[3] * maxprim + pc.zb];
                double wt[16];
                for (int m = 0; m < 16; ++m) {
                    double x = 1.0;
                    for (int c = 0; c < 4; ++c)
                        if (m & (1 << c)) x *= w[c];
                    wt[m] = x;
                }
                const int* tg = pl.target.data();
                const uint8_t* wp = pl.wpat.data();
                for (int n = 0; n < ncart4; ++n) acc[n] += wt[wp[n]] * v[tg[n]];
            }
        }
        // Cartesian -> spherical for d shells
        int nf[4] = {nfunc(t[0]), nfunc(t[1]), nfunc(t[2]), nfunc(t[3])};
        cur.assign(acc.begin(), acc.end());
        int dims[4] = {nc[0], nc[1], nc[2], nc[3]};
        for (int c = 0; c < 4; ++c) {
            if (t[c] != HFGPU_SHELL_D) continue;
            int outer = 1, inner = 1;
            for (int q = 0; q < c; ++q) outer *= dims[q];
            for (int q = c + 1; q < 4; ++q) inner *= dims[q];
            nx.assign((size_t)outer * 5 * inner, 0.0);
            for (int o = 0; o < outer; ++o)
                for (int sidx = 0; sidx < 5; ++sidx)
                    for (int cc = 0; cc < 6; ++cc) {
                        double h = harm(sidx, cc);
                        if (h == 0) continue;
                        for (int in = 0; in < inner; ++in)
                            nx[((size_t)o * 5 + sidx) * inner + in] += h * cur[((size_t)o * 6 + cc) * inner + in];
                    }
            cur.swap(nx);
            dims[c] = 5;
        }
        int nout = nf[0] * nf[1] * nf[2] * nf[3];
        std::memcpy(out, cur.data(), sizeof(double) * nout);
    }

    // One-electron integrals S, T, V (cmpt1e.f90 with one_electron_terms.f90:
    // s_s_1e_terms ... d_l_1e_terms): every primitive pair of every shell
    // pair (no negab screen there), coefficients djk_a*djk_b with the L-shell
    // p/s ratio djkl on p components, the Boys routine of the pair's total
    // angular momentum (boys_0/1/2/n as each *_1e_terms routine calls it),
    // Cartesian d transformed with matharmond.  Obara-Saika recurrences:
    //   overlap    s(i+1,j) = PA s(i,j) + (i s(i-1,j) + j s(i,j-1))/2p, per axis
    //   kinetic    t(i,j) = -2b^2 s(i,j+2) + b(2j+1) s(i,j) - j(j-1)/2 s(i,j-2)
    //   nuclear    V(a+1,b)^m = PA V(a,b)^m - PC V(a,b)^(m+1)
    //                          + a/2p (V(a-1,b)^m - V(a-1,b)^(m+1)) + b/2p (...)
    //              V(0,0)^m = 2 pi/p exp(-ab/p AB^2) F_m(p PC^2)
    // S, T, V are nb x nb, symmetric, written in full.
    void one_electron(int natom, const double* Z, const double* xyz, double* S, double* T, double* V) {
        const size_t nb2 = (size_t)nb * nb;
        std::fill(S, S + nb2, 0.0);
        std::fill(T, T + nb2, 0.0);
        std::fill(V, V + nb2, 0.0);
        std::vector<std::pair<int, int>> plist;
        for (int a = 0; a < nsh; ++a)
            for (int b = 0; b <= a; ++b) plist.push_back({a, b});
#pragma omp parallel for schedule(dynamic)
        for (long long ip = 0; ip < (long long)plist.size(); ++ip) {
            const int a = plist[ip].first, b = plist[ip].second;
            const int ta = shtyp[a], tb = shtyp[b];
            const int na = ncart(ta), nbc = ncart(tb);
            const Cart* ca = carts(ta);
            const Cart* cb = carts(tb);
            const int la = lmax(ta), lb = lmax(tb), nboys = la + lb;
            double cs[6][6] = {}, ct[6][6] = {}, cv[6][6] = {};
            const double* A = &xsh[3 * a];
            const double* B = &xsh[3 * b];
            double ab2 = 0;
            for (int x = 0; x < 3; ++x) ab2 += (A[x] - B[x]) * (A[x] - B[x]);
            for (int za = 0; za < nzet[a]; ++za)
                for (int zb = 0; zb < nzet[b]; ++zb) {
                    const double ea = zeta[(size_t)a * maxprim + za], eb = zeta[(size_t)b * maxprim + zb];
                    const double p = ea + eb, op = 1.0 / p, mu = ea * eb * op;
                    const double dd = djk[(size_t)a * maxprim + za] * djk[(size_t)b * maxprim + zb];
                    const double ga = djkl[(size_t)a * maxprim + za], gb = djkl[(size_t)b * maxprim + zb];
                    const double K = std::exp(-mu * ab2);
                    double P[3], PA[3], PB[3];
                    for (int x = 0; x < 3; ++x) {
                        P[x] = (ea * A[x] + eb * B[x]) * op;
                        PA[x] = P[x] - A[x];
                        PB[x] = P[x] - B[x];
                    }
                    // 1D overlap tables s[x][i][j], i <= la, j <= lb + 2
                    double s1[3][3][5];
                    for (int x = 0; x < 3; ++x) {
                        for (int i = 0; i < 3; ++i)
                            for (int j = 0; j < 5; ++j) s1[x][i][j] = 0.0;
                        s1[x][0][0] = 1.0;
                        for (int j = 0; j < 4; ++j)
                            s1[x][0][j + 1] = PB[x] * s1[x][0][j] + (j > 0 ? 0.5 * op * j * s1[x][0][j - 1] : 0.0);
                        for (int i = 0; i < 2; ++i)
                            for (int j = 0; j < 5; ++j) {
                                double v = PA[x] * s1[x][i][j];
                                if (i > 0) v += 0.5 * op * i * s1[x][i - 1][j];
                                if (j > 0) v += 0.5 * op * j * s1[x][i][j - 1];
                                s1[x][i + 1][j] = v;
                            }
                    }
                    const double s00 = std::pow(PI * op, 1.5) * K;
                    auto t1 = [&](int x, int i, int j) {
                        double v = -2.0 * eb * eb * s1[x][i][j + 2] + eb * (2 * j + 1) * s1[x][i][j];
                        if (j >= 2) v -= 0.5 * j * (j - 1) * s1[x][i][j - 2];
                        return v;
                    };
                    // nuclear attraction: V[a][b][m] over Cartesian exponents
                    // (la, lb <= 2 -> exponent vectors indexed 0..26)
                    double vn[6][6] = {};
                    for (int nuc = 0; nuc < natom; ++nuc) {
                        double PC[3], pc2 = 0;
                        for (int x = 0; x < 3; ++x) {
                            PC[x] = P[x] - xyz[3 * nuc + x];
                            pc2 += PC[x] * PC[x];
                        }
                        double fm[16];
                        boys(nboys, p * pc2, fm);
                        // memo[ia][ib][m], ia/ib = exponent index ex*9+ey*3+ez
                        const double base = 2.0 * PI * op * K;
                        std::function<double(int, int, int, int, int, int, int)> rec;
                        double memo[27][27][5];
                        bool done[27][27][5] = {};
                        rec = [&](int ax, int ay, int az, int bx, int by, int bz, int m) -> double {
                            if (ax < 0 || ay < 0 || az < 0 || bx < 0 || by < 0 || bz < 0) return 0.0;
                            const int ia = ax * 9 + ay * 3 + az, ib = bx * 9 + by * 3 + bz;
                            if (done[ia][ib][m]) return memo[ia][ib][m];
                            double r;
                            int av[3] = {ax, ay, az}, bv[3] = {bx, by, bz};
                            if (ax + ay + az > 0) {
                                int i = ax > 0 ? 0 : ay > 0 ? 1 : 2;
                                av[i] -= 1;
                                r = PA[i] * rec(av[0], av[1], av[2], bx, by, bz, m) -
                                    PC[i] * rec(av[0], av[1], av[2], bx, by, bz, m + 1);
                                if (av[i] > 0) {
                                    int a2[3] = {av[0], av[1], av[2]};
                                    a2[i] -= 1;
                                    r += 0.5 * op * av[i] *
                                         (rec(a2[0], a2[1], a2[2], bx, by, bz, m) - rec(a2[0], a2[1], a2[2], bx, by, bz, m + 1));
                                }
                                if (bv[i] > 0) {
                                    int b2[3] = {bx, by, bz};
                                    b2[i] -= 1;
                                    r += 0.5 * op * bv[i] *
                                         (rec(av[0], av[1], av[2], b2[0], b2[1], b2[2], m) -
                                          rec(av[0], av[1], av[2], b2[0], b2[1], b2[2], m + 1));
                                }
                            } else if (bx + by + bz > 0) {
                                int i = bx > 0 ? 0 : by > 0 ? 1 : 2;
                                bv[i] -= 1;
                                r = PB[i] * rec(0, 0, 0, bv[0], bv[1], bv[2], m) -
                                    PC[i] * rec(0, 0, 0, bv[0], bv[1], bv[2], m + 1);
                                if (bv[i] > 0) {
                                    int b2[3] = {bv[0], bv[1], bv[2]};
                                    b2[i] -= 1;
                                    r += 0.5 * op * bv[i] *
                                         (rec(0, 0, 0, b2[0], b2[1], b2[2], m) - rec(0, 0, 0, b2[0], b2[1], b2[2], m + 1));
                                }
                            } else {
                                r = base * fm[m];
                            }
                            done[ia][ib][m] = true;
                            memo[ia][ib][m] = r;
                            return r;
                        };
                        for (int i = 0; i < na; ++i)
                            for (int j = 0; j < nbc; ++j)
                                vn[i][j] -= Z[nuc] * rec(ca[i].x, ca[i].y, ca[i].z, cb[j].x, cb[j].y, cb[j].z, 0);
                    }
                    for (int i = 0; i < na; ++i)
                        for (int j = 0; j < nbc; ++j) {
                            double w = dd;
                            if (ta == HFGPU_SHELL_L && ca[i].x + ca[i].y + ca[i].z == 1) w *= ga;
                            if (tb == HFGPU_SHELL_L && cb[j].x + cb[j].y + cb[j].z == 1) w *= gb;
                            const int ix = ca[i].x, iy = ca[i].y, iz = ca[i].z;
                            const int jx = cb[j].x, jy = cb[j].y, jz = cb[j].z;
                            const double sx = s1[0][ix][jx], sy = s1[1][iy][jy], sz = s1[2][iz][jz];
                            cs[i][j] += w * s00 * sx * sy * sz;
                            ct[i][j] += w * s00 * (t1(0, ix, jx) * sy * sz + sx * t1(1, iy, jy) * sz + sx * sy * t1(2, iz, jz));
                            cv[i][j] += w * vn[i][j];
                        }
                }
            // Cartesian -> spherical d (matharmond) on each d side
            const int fa = nfunc(ta), fb = nfunc(tb);
            double* mats[3] = {&cs[0][0], &ct[0][0], &cv[0][0]};
            double* outs[3] = {S, T, V};
            for (int k = 0; k < 3; ++k) {
                double (*m)[6] = (double (*)[6])mats[k];
                double r1[6][6] = {};
                for (int i = 0; i < fa; ++i)
                    for (int j = 0; j < nbc; ++j) {
                        if (ta == HFGPU_SHELL_D) {
                            double x = 0;
                            for (int c = 0; c < 6; ++c) x += harm(i, c) * m[c][j];
                            r1[i][j] = x;
                        } else {
                            r1[i][j] = m[i][j];
                        }
                    }
                for (int i = 0; i < fa; ++i)
                    for (int j = 0; j < fb; ++j) {
                        double x;
                        if (tb == HFGPU_SHELL_D) {
                            x = 0;
                            for (int c = 0; c < 6; ++c) x += harm(j, c) * r1[i][c];
                        } else {
                            x = r1[i][j];
                        }
                        const size_t r = (size_t)aosh[a] + i, c = (size_t)aosh[b] + j;
                        outs[k][c * nb + r] = x;
                        outs[k][r * nb + c] = x;
                    }
            }
        }
    }

    int nfunc_pair(int pid) const { return nfunc(shtyp[pairs[pid].sh1]) * nfunc(shtyp[pairs[pid].sh2]); }

    // evaluate_maxdm.f90:1-101, by pair id (incl. the d-l block as written there)
    void maxdm(const double* P, std::vector<double>& md) {
        md.assign(pairs.size(), 0.0);
        for (size_t id = 0; id < pairs.size(); ++id) {
            int a = pairs[id].sh1, b = pairs[id].sh2;
            int ta = shtyp[a], tb = shtyp[b];
            int r0 = aosh[a], c0 = aosh[b];
            int nr = nfunc(ta), nc_ = nfunc(tb);
            if (ta == HFGPU_SHELL_D && tb == HFGPU_SHELL_L) { nr = 4; nc_ = 5; }
            double m = 0;
            for (int i = 0; i < nr; ++i)
                for (int j = 0; j < nc_; ++j) {
                    int row = r0 + i, col = c0 + j;
                    if (row >= nb || col >= nb) continue;  // out of range in the reference too
                    m = std::max(m, std::fabs(P[(size_t)col * nb + row]));
                }
            md[id] = m;
        }
    }

    // Element-level scatter of one ERI block into G with weight s.
    // jk: 0 = J and K, 1 = J only.  thr_elem > 0 -> skip |v| <= thr_elem.
    void scatter(int pab, int pcd, const double* e, double s, const double* P, double* G,
                 double thr_elem, int jonly) {
        int a = pairs[pab].sh1, b = pairs[pab].sh2, c = pairs[pcd].sh1, d = pairs[pcd].sh2;
        int na = nfunc(shtyp[a]), nbb = nfunc(shtyp[b]), nc_ = nfunc(shtyp[c]), nd = nfunc(shtyp[d]);
        int n = 0;
        auto Pm = [&](int i, int j) { return P[(size_t)j * nb + i]; };
        for (int i = 0; i < na; ++i) for (int j = 0; j < nbb; ++j)
        for (int k = 0; k < nc_; ++k) for (int l = 0; l < nd; ++l, ++n) {
            double v = e[n];
            if (thr_elem > 0 && !(std::fabs(v) > thr_elem)) continue;
            int I = aosh[a] + i, J = aosh[b] + j, K = aosh[c] + k, L = aosh[d] + l;
            G[(size_t)J * nb + I] += 2 * s * Pm(K, L) * v;
            G[(size_t)L * nb + K] += 2 * s * Pm(I, J) * v;
            if (jonly) continue;
            double h = 0.5 * s * v;
            G[(size_t)K * nb + I] -= h * Pm(J, L);
            G[(size_t)L * nb + I] -= h * Pm(J, K);
            G[(size_t)K * nb + J] -= h * Pm(I, L);
            G[(size_t)L * nb + J] -= h * Pm(I, K);
        }
    }

    static void add_sym(double* F, const double* G, int nb) {
        for (int j = 0; j < nb; ++j)
            for (int i = 0; i < nb; ++i)
                F[(size_t)j * nb + i] += G[(size_t)j * nb + i] + G[(size_t)i * nb + j];
    }

    double diag_weight(int pid) const { double f = pairs[pid].sh1 == pairs[pid].sh2 ? 1.0 : 2.0; return f * f / 8.0; }

    void initial_diag(double* F, const double* P, double thr) {
        (void)thr;  // used by the reference only for its (pp|pp) class
        std::vector<double> G((size_t)nb * nb, 0.0);
        std::vector<double> e(625);
        for (int c = 0; c < NCLASS; ++c) {
            for (int id : cls[c]) {
                eri(id, id, e.data());
                int n = nfunc_pair(id) * nfunc_pair(id);
                double mx = 0;
                for (int q = 0; q < n; ++q) mx = std::max(mx, std::fabs(e[q]));
                schw[id] = std::sqrt(mx);
                double th = INTTHRESH;
                if (c == CPP) th = thr;  // fock_build_initial_diag.f90:277 uses thr for (pp|pp)
                scatter(id, id, e.data(), diag_weight(id), P, G.data(), th, 0);
            }
        }
        add_sym(F, G.data(), nb);
        sort_schwarz();
    }

    // index_sort + find_threshold (index_sort.f90): descending by schw,
    // ties by list position; last = first position (1-based) below shthresh.
    void sort_schwarz() {
        for (int c = 0; c < NCLASS; ++c) {
            int n = (int)cls[c].size();
            std::vector<int> ord(n);
            std::iota(ord.begin(), ord.end(), 0);
            std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return schw[cls[c][x]] > schw[cls[c][y]]; });
            order[c].resize(n);
            for (int i = 0; i < n; ++i) order[c][i] = cls[c][ord[i]];
            if (n == 0) { last[c] = 0; continue; }
            if (schw[order[c][0]] < SHTHRESH) { last[c] = 1; continue; }
            if (schw[order[c][n - 1]] > SHTHRESH) { last[c] = n; continue; }
            last[c] = n;
            for (int i = 0; i < n; ++i)
                if (schw[order[c][i]] < SHTHRESH) { last[c] = i + 1; break; }
        }
        have_schwarz = true;
    }

    void diag(double* F, const double* P, double thr) {
        std::vector<double> md;
        maxdm(P, md);
        std::vector<double> G((size_t)nb * nb, 0.0);
        std::vector<double> e(625);
        for (int c = 0; c < NCLASS; ++c)
            for (int id : cls[c]) {
                int a = pairs[id].sh1, b = pairs[id].sh2;
                double mv = std::max(md[id], std::max(.25 * md[pairid[(size_t)b * nsh + b]], .25 * md[pairid[(size_t)a * nsh + a]]));
                if (schw[id] * schw[id] * mv < thr) continue;
                eri(id, id, e.data());
                if (c == CPP) {  // fock_build_diag.f90:176 whole-quartet skip for (pp|pp)
                    int n = nfunc_pair(id) * nfunc_pair(id);
                    double mx = 0;
                    for (int q = 0; q < n; ++q) mx = std::max(mx, std::fabs(e[q]));
                    if (mx < thr) continue;
                }
                scatter(id, id, e.data(), diag_weight(id), P, G.data(), INTTHRESH, 0);
            }
        add_sym(F, G.data(), nb);
    }

    void non_diag(double* F, const double* P, double thr, int jonly, int stride = 1, int offset = 0) {
        std::vector<double> md;
        maxdm(P, md);
        std::vector<double> G((size_t)nb * nb, 0.0);
        std::fill(class_pass.begin(), class_pass.end(), 0);
        std::fill(class_scatter.begin(), class_scatter.end(), 0);
        for (int ca = 0; ca < NCLASS; ++ca)
            for (int cb = ca; cb < NCLASS; ++cb) {
                int la = last[ca], lb = last[cb];
                if (la == 0 || lb == 0) continue;
                long long npass = 0, nscat = 0;
#pragma omp parallel reduction(+ : npass, nscat)
                {
                    std::vector<double> Gl((size_t)nb * nb, 0.0);
                    std::vector<double> e(625);
#pragma omp for schedule(dynamic)
                    for (int ii = (ca == cb ? 1 : 0); ii < la; ++ii) {
                        if (ii % stride != offset) continue;  // bounded CPU-baseline sample
                        int p1 = order[ca][ii];
                        int s1 = pairs[p1].sh1, s2 = pairs[p1].sh2;
                        int jend = (ca == cb) ? ii : lb;
                        for (int jj = 0; jj < jend; ++jj) {
                            int p2 = order[cb][jj];
                            int s3 = pairs[p2].sh1, s4 = pairs[p2].sh2;
                            double dc = std::max(md[p1], md[p2]);
                            double sc;
                            if (jonly) {
                                sc = dc;
                            } else {
                                double dx = std::max(std::max(md[pairid[(size_t)s1 * nsh + s3]], md[pairid[(size_t)s1 * nsh + s4]]),
                                                     std::max(md[pairid[(size_t)s2 * nsh + s3]], md[pairid[(size_t)s2 * nsh + s4]]));
                                sc = std::max(dc, .25 * dx);
                            }
                            if (schw[p1] * schw[p2] * sc < thr) continue;
                            ++npass;
                            eri(p1, p2, e.data());
                            int n = nfunc_pair(p1) * nfunc_pair(p2);
                            double mx = 0;
                            for (int q = 0; q < n; ++q) mx = std::max(mx, std::fabs(e[q]));
                            if (mx < thr) continue;
                            ++nscat;
                            double s = (s1 == s2 ? 1.0 : 2.0) * (s3 == s4 ? 1.0 : 2.0) * 2.0 / 8.0;
                            scatter(p1, p2, e.data(), s, P, Gl.data(), 0.0, jonly);
                        }
                    }
#pragma omp critical
                    for (size_t q = 0; q < G.size(); ++q) G[q] += Gl[q];
                }
                class_pass[ca * NCLASS + cb] = npass;
                class_scatter[ca * NCLASS + cb] = nscat;
            }
        n_screen_pass = 0; n_scatter = 0;
        for (int q = 0; q < NCLASS * NCLASS; ++q) { n_screen_pass += class_pass[q]; n_scatter += class_scatter[q]; }
        add_sym(F, G.data(), nb);
    }
};

}  // namespace

extern "C" {

void* orc_create(const hfgpu_basis* b) {
    Oracle* o = new Oracle();
    o->init(b);
    return o;
}
void orc_destroy(void* h) { delete (Oracle*)h; }

void orc_boys(int n, double x, double* fn) { boys(n, x, fn); }

int orc_npairs(void* h) { return (int)((Oracle*)h)->pairs.size(); }

// Contracted ERI block of the shell quartet (s1 s2|s3 s4) in the given
// shell order (0-based shells); returns the number of values written.
int orc_eri(void* h, int s1, int s2, int s3, int s4, double* out) {
    Oracle* o = (Oracle*)h;
    // build ad-hoc pairs in the requested order, with the negab screen
    auto mk = [&](int a, int b) {
        PairData pd; pd.sh1 = a; pd.sh2 = b;
        double r2 = 0;
        for (int x = 0; x < 3; ++x) { double d = o->xsh[3 * a + x] - o->xsh[3 * b + x]; r2 += d * d; }
        for (int za = 0; za < o->nzet[a]; ++za)
            for (int zb = 0; zb < o->nzet[b]; ++zb) {
                double ea = o->zeta[(size_t)a * o->maxprim + za], eb = o->zeta[(size_t)b * o->maxprim + zb];
                double p = ea + eb, pm1 = 1.0 / p, q = ea * eb * pm1;
                double dd = o->djk[(size_t)a * o->maxprim + za] * o->djk[(size_t)b * o->maxprim + zb];
                double K = RT2PI54 * std::exp(-q * r2) * pm1 * dd;
                if (std::fabs(K) * std::sqrt(pm1) < EXTRATHRESH) continue;
                PrimPair pp{p, (ea * o->xsh[3 * a] + eb * o->xsh[3 * b]) * pm1,
                            (ea * o->xsh[3 * a + 1] + eb * o->xsh[3 * b + 1]) * pm1,
                            (ea * o->xsh[3 * a + 2] + eb * o->xsh[3 * b + 2]) * pm1, K, za, zb};
                pd.prims.push_back(pp);
            }
        return pd;
    };
    size_t base = o->pairs.size();
    o->pairs.push_back(mk(s1, s2));
    o->pairs.push_back(mk(s3, s4));
    o->eri((int)base, (int)base + 1, out);
    int n = nfunc(o->shtyp[s1]) * nfunc(o->shtyp[s2]) * nfunc(o->shtyp[s3]) * nfunc(o->shtyp[s4]);
    o->pairs.resize(base);
    return n;
}

void orc_fock_build_initial_diag(void* h, double* f, const double* p, double thr) {
    ((Oracle*)h)->initial_diag(f, p, thr);
}
int orc_fock_build_diag(void* h, double* f, const double* p, double thr) {
    Oracle* o = (Oracle*)h;
    if (!o->have_schwarz) return 1;
    o->diag(f, p, thr);
    return 0;
}
int orc_fock_build_non_diag(void* h, double* f, const double* p, double thr) {
    Oracle* o = (Oracle*)h;
    if (!o->have_schwarz) return 1;
    o->non_diag(f, p, thr, 0);
    return 0;
}
int orc_fock_build_non_diag_j_only(void* h, double* f, const double* p, double thr) {
    Oracle* o = (Oracle*)h;
    if (!o->have_schwarz) return 1;
    o->non_diag(f, p, thr, 1);
    return 0;
}

// Sampled off-diagonal build for the CPU baseline: only bra rows
// ii % stride == offset of every class block; returns the screened-in count.
long long orc_fock_build_non_diag_sample(void* h, double* f, const double* p, double thr, int stride, int offset) {
    Oracle* o = (Oracle*)h;
    if (!o->have_schwarz) return -1;
    o->non_diag(f, p, thr, 0, stride, offset);
    return o->n_screen_pass;
}

// Schwarz state left by fock_build_initial_diag: schw by (sh1,sh2) in an
// nsh x nsh matrix, and last[10] per class (ss sp sd sl pp pd pl dd dl ll).
void orc_schwarz(void* h, double* schw_sh, int* last) {
    Oracle* o = (Oracle*)h;
    for (int a = 0; a < o->nsh; ++a)
        for (int b = 0; b < o->nsh; ++b)
            schw_sh[(size_t)a * o->nsh + b] = o->schw[o->pairid[(size_t)a * o->nsh + b]];
    for (int c = 0; c < NCLASS; ++c) last[c] = o->last[c];
}

// Quartet counts of the last non-diag build: [10][10] screen-pass and
// post-screen-pass counts per (bra class, ket class).
void orc_counts(void* h, long long* pass, long long* scat) {
    Oracle* o = (Oracle*)h;
    for (int q = 0; q < NCLASS * NCLASS; ++q) { pass[q] = o->class_pass[q]; scat[q] = o->class_scatter[q]; }
}

void orc_maxdm(void* h, const double* p, double* md_sh) {
    Oracle* o = (Oracle*)h;
    std::vector<double> md;
    o->maxdm(p, md);
    for (int a = 0; a < o->nsh; ++a)
        for (int b = 0; b < o->nsh; ++b)
            md_sh[(size_t)a * o->nsh + b] = md[o->pairid[(size_t)a * o->nsh + b]];
}

// One-electron integrals S, T, V (nb x nb, symmetric) for natom nuclei of
// charges Z at xyz (bohr, row per atom).
void orc_one_electron(void* h, int natom, const double* Z, const double* xyz, double* S, double* T, double* V) {
    ((Oracle*)h)->one_electron(natom, Z, xyz, S, T, V);
}

int orc_num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
