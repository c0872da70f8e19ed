// One-electron integrals on the host: overlap S, kinetic T and nuclear
// attraction V over the same contracted shells as the Fock builder.
//
// The reference computes these once per job in cmpt1e.f90 with the
// per-class routines of one_electron_terms.f90; they are O(N^2) set-up, off
// the Fock-build hot path.  Here they are restated with the Obara-Saika
// recurrences: 1D overlap S_{i,j} for the Gaussian product, the kinetic
// integral as 1/2 <di/dx|dj/dx> per direction, and the nuclear attraction
// through the [a|A(0)|b]^(m) recurrence seeded with the Boys function.
// Contraction, L-shell p/s ratios and the spherical d transform follow the
// same conventions as the ERIs (read_basfile.f90:100-179,
// spread_basis.f90:149-151, index_functions.f90:147-168).
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "../../include/hfgpu.h"

namespace {

const double PI = 3.141592653589793238462643383279502884197;
#define PI_D 3.141592653589793238462643383279502884197

struct C3 { int x, y, z; };

void carts_of(int t, std::vector<C3>& c, std::vector<int>& isp) {
    c.clear(); isp.clear();
    if (t == HFGPU_SHELL_S || t == HFGPU_SHELL_L) { c.push_back({0, 0, 0}); isp.push_back(0); }
    if (t == HFGPU_SHELL_P || t == HFGPU_SHELL_L) {
        c.push_back({1, 0, 0}); c.push_back({0, 1, 0}); c.push_back({0, 0, 1});
        for (int i = 0; i < 3; ++i) isp.push_back(t == HFGPU_SHELL_L ? 1 : 0);
    }
    if (t == HFGPU_SHELL_D) {
        const C3 d[6] = {{2, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 2, 0}, {0, 1, 1}, {0, 0, 2}};
        for (int i = 0; i < 6; ++i) { c.push_back(d[i]); isp.push_back(0); }
    }
}

int nfunc_of(int t) { return t == HFGPU_SHELL_S ? 1 : t == HFGPU_SHELL_P ? 3 : t == HFGPU_SHELL_D ? 5 : 4; }

// F_m(T), m = 0..n, to ~1e-15: series below 30, asymptotic + upward above.
__host__ __device__ void boys_acc(int n, double T, double* F) {
    if (T < 30.0) {
        // F_n by its series, then downward recursion
        double term = 1.0 / (2 * n + 1), sum = term;
        for (int k = 1; k < 300; ++k) {
            term *= 2.0 * T / (2 * n + 2 * k + 1);
            sum += term;
            if (term < 1e-17 * sum) break;
        }
        double e = exp(-T);
        F[n] = e * sum;
        for (int m = n - 1; m >= 0; --m) F[m] = (2.0 * T * F[m + 1] + e) / (2 * m + 1);
    } else {
        F[0] = 0.5 * sqrt(PI_D / T) * erf(sqrt(T));
        double e = exp(-T);
        for (int m = 0; m < n; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) / (2.0 * T);
    }
}

const double SQ3 = 1.7320508075688772935;
// spherical d (z2, xz, yz, xy, x2-y2) from Cartesian (xx,xy,xz,yy,yz,zz)
const double HARM[5][6] = {{-.5, 0, 0, -.5, 0, 1.0}, {0, 0, SQ3, 0, 0, 0}, {0, 0, 0, 0, SQ3, 0},
                           {0, SQ3, 0, 0, 0, 0}, {SQ3 / 2, 0, 0, -SQ3 / 2, 0, 0}};

// transform the Cartesian block (na x nb) of a shell pair to the function block
void to_functions(int ta, int tb, const std::vector<double>& cart, int nca, int ncb, std::vector<double>& out) {
    int nfa = nfunc_of(ta), nfb = nfunc_of(tb);
    std::vector<double> tmp((size_t)nfa * ncb, 0.0);
    for (int j = 0; j < ncb; ++j) {
        if (ta == HFGPU_SHELL_D) {
            for (int s = 0; s < 5; ++s) {
                double v = 0;
                for (int c = 0; c < 6; ++c) v += HARM[s][c] * cart[(size_t)c * ncb + j];
                tmp[(size_t)s * ncb + j] = v;
            }
        } else {
            for (int i = 0; i < nca; ++i) tmp[(size_t)i * ncb + j] = cart[(size_t)i * ncb + j];
        }
    }
    out.assign((size_t)nfa * nfb, 0.0);
    for (int i = 0; i < nfa; ++i) {
        if (tb == HFGPU_SHELL_D) {
            for (int s = 0; s < 5; ++s) {
                double v = 0;
                for (int c = 0; c < 6; ++c) v += HARM[s][c] * tmp[(size_t)i * ncb + c];
                out[(size_t)i * nfb + s] = v;
            }
        } else {
            for (int j = 0; j < ncb; ++j) out[(size_t)i * nfb + j] = tmp[(size_t)i * ncb + j];
        }
    }
}

// 1D overlap table S[i][j], i <= la+1, j <= lb+1 (Obara-Saika)
__host__ __device__ void overlap_1d(double PA, double PB, double p, int la, int lb, double S[5][5]) {
    const double h = 0.5 / p;
    for (int i = 0; i <= la; ++i)
        for (int j = 0; j <= lb; ++j) S[i][j] = 0.0;
    S[0][0] = 1.0;
    for (int i = 0; i <= la; ++i)
        for (int j = 0; j <= lb; ++j) {
            if (i == 0 && j == 0) continue;
            double v;
            if (i > 0) {
                v = PA * S[i - 1][j];
                if (i > 1) v += h * (i - 1) * S[i - 2][j];
                if (j > 0) v += h * j * S[i - 1][j - 1];
            } else {
                v = PB * S[i][j - 1];
                if (j > 1) v += h * (j - 1) * S[i][j - 2];
            }
            S[i][j] = v;
        }
}

// Nuclear attraction [a|C|b]^(m) by Obara-Saika on the bra, then the ket.
// The recurrence tree depends only on the Cartesian components, so it is
// compiled once per (la, lb) into a flat list of ops evaluated per primitive
// pair and nucleus.
struct NucOp { int kind, ax, m, c0, c1, c2, c3, c4, c5, n1, n2; };
// kind 0: base F[m]; 1: bra step; 2: ket step
struct NucPlan {
    std::vector<NucOp> ops;
    std::vector<int> target;  // per (i,j) Cartesian pair
    std::map<long long, int> idx;
    static long long key(const int* a, const int* b, int m) {
        long long k = m;
        for (int i = 0; i < 3; ++i) k = k * 8 + a[i];
        for (int i = 0; i < 3; ++i) k = k * 8 + b[i];
        return k;
    }
    int get(const int* a, const int* b, int m) {
        long long k = key(a, b, m);
        auto it = idx.find(k);
        if (it != idx.end()) return it->second;
        NucOp op{0, 0, m, -1, -1, -1, -1, -1, -1, 0, 0};
        int ax = -1;
        for (int i = 0; i < 3; ++i) if (a[i] > 0) { ax = i; break; }
        if (ax >= 0) {
            int a1[3] = {a[0], a[1], a[2]}; a1[ax]--;
            op.kind = 1; op.ax = ax;
            op.c0 = get(a1, b, m); op.c1 = get(a1, b, m + 1);
            if (a1[ax] > 0) {
                int a2[3] = {a1[0], a1[1], a1[2]}; a2[ax]--;
                op.n1 = a1[ax]; op.c2 = get(a2, b, m); op.c3 = get(a2, b, m + 1);
            }
            if (b[ax] > 0) {
                int b1[3] = {b[0], b[1], b[2]}; b1[ax]--;
                op.n2 = b[ax]; op.c4 = get(a1, b1, m); op.c5 = get(a1, b1, m + 1);
            }
        } else {
            int bx = -1;
            for (int i = 0; i < 3; ++i) if (b[i] > 0) { bx = i; break; }
            if (bx >= 0) {
                int b1[3] = {b[0], b[1], b[2]}; b1[bx]--;
                op.kind = 2; op.ax = bx;
                op.c0 = get(a, b1, m); op.c1 = get(a, b1, m + 1);
                if (b1[bx] > 0) {
                    int b2[3] = {b1[0], b1[1], b1[2]}; b2[bx]--;
                    op.n1 = b1[bx]; op.c2 = get(a, b2, m); op.c3 = get(a, b2, m + 1);
                }
            }
        }
        int id = (int)ops.size();
        ops.push_back(op);
        idx[k] = id;
        return id;
    }
    void eval(const double* PA, const double* PB, const double* PC, double h, const double* F,
              std::vector<double>& v) const {
        v.resize(ops.size());
        for (size_t o = 0; o < ops.size(); ++o) {
            const NucOp& op = ops[o];
            double x;
            if (op.kind == 0) {
                x = F[op.m];
            } else {
                const double g = op.kind == 1 ? PA[op.ax] : PB[op.ax];
                x = g * v[op.c0] - PC[op.ax] * v[op.c1];
                if (op.n1) x += h * op.n1 * (v[op.c2] - v[op.c3]);
                if (op.n2) x += h * op.n2 * (v[op.c4] - v[op.c5]);
            }
            v[o] = x;
        }
    }
};

}  // namespace

extern "C" int hfgpu_one_electron(const hfgpu_basis* B, int natom, const double* charges, const double* xyz,
                                  double* S, double* T, double* V) {
    if (!B || B->nsh <= 0) return HFGPU_ERR_ARG;
    const int nb = B->nb, MP = B->maxprim;
    if (S) std::memset(S, 0, sizeof(double) * nb * nb);
    if (T) std::memset(T, 0, sizeof(double) * nb * nb);
    if (V) std::memset(V, 0, sizeof(double) * nb * nb);
    std::vector<C3> ca, cb;
    std::vector<int> ia, ib;
    for (int a = 0; a < B->nsh; ++a)
        for (int b = 0; b <= a; ++b) {
            int ta = B->shtyp[a], tb = B->shtyp[b];
            carts_of(ta, ca, ia);
            carts_of(tb, cb, ib);
            const int na = (int)ca.size(), nbb = (int)cb.size();
            std::vector<double> s((size_t)na * nbb, 0.0), t((size_t)na * nbb, 0.0), v((size_t)na * nbb, 0.0);
            const double* A = B->xsh + 3 * a;
            const double* Bc = B->xsh + 3 * b;
            double AB2 = 0;
            for (int x = 0; x < 3; ++x) AB2 += (A[x] - Bc[x]) * (A[x] - Bc[x]);
            NucPlan plan;
            for (int i = 0; i < na; ++i)
                for (int j = 0; j < nbb; ++j) {
                    int ai[3] = {ca[i].x, ca[i].y, ca[i].z}, bj[3] = {cb[j].x, cb[j].y, cb[j].z};
                    plan.target.push_back(plan.get(ai, bj, 0));
                }
            std::vector<double> work;
            const int la = ta == HFGPU_SHELL_D ? 2 : ta == HFGPU_SHELL_S ? 0 : 1;
            const int lb = tb == HFGPU_SHELL_D ? 2 : tb == HFGPU_SHELL_S ? 0 : 1;
            for (int za = 0; za < B->nzet[a]; ++za)
                for (int zb = 0; zb < B->nzet[b]; ++zb) {
                    const double ea = B->zeta[(size_t)a * MP + za], eb = B->zeta[(size_t)b * MP + zb];
                    const double p = ea + eb, mu = ea * eb / p;
                    double P[3], PA[3], PB[3];
                    for (int x = 0; x < 3; ++x) {
                        P[x] = (ea * A[x] + eb * Bc[x]) / p;
                        PA[x] = P[x] - A[x];
                        PB[x] = P[x] - Bc[x];
                    }
                    const double K = std::exp(-mu * AB2);
                    const double da = B->djk[(size_t)a * MP + za], db = B->djk[(size_t)b * MP + zb];
                    const double ra = ta == HFGPU_SHELL_L ? B->djkl[(size_t)a * MP + za] : 1.0;
                    const double rb = tb == HFGPU_SHELL_L ? B->djkl[(size_t)b * MP + zb] : 1.0;
                    double s1[3][5][5];
                    for (int x = 0; x < 3; ++x) overlap_1d(PA[x], PB[x], p, la + 1, lb + 1, s1[x]);
                    const double pre = std::pow(PI / p, 1.5) * K;
                    // nuclear attraction base values per centre
                    std::vector<double> vv((size_t)na * nbb, 0.0);
                    if (V) {
                        const int L = la + lb;
                        double Fm[16], base[16], PC[3];
                        for (int c = 0; c < natom; ++c) {
                            double PC2 = 0;
                            for (int x = 0; x < 3; ++x) {
                                PC[x] = P[x] - xyz[3 * c + x];
                                PC2 += PC[x] * PC[x];
                            }
                            boys_acc(L, p * PC2, Fm);
                            for (int m = 0; m <= L; ++m) base[m] = 2.0 * PI / p * K * Fm[m];
                            plan.eval(PA, PB, PC, 0.5 / p, base, work);
                            for (int q = 0; q < na * nbb; ++q) vv[q] -= charges[c] * work[plan.target[q]];
                        }
                    }
                    for (int i = 0; i < na; ++i)
                        for (int j = 0; j < nbb; ++j) {
                            const int e1[3] = {ca[i].x, ca[i].y, ca[i].z}, e2[3] = {cb[j].x, cb[j].y, cb[j].z};
                            double w = da * db * (ia[i] ? ra : 1.0) * (ib[j] ? rb : 1.0);
                            double sx[3], tx[3];
                            for (int x = 0; x < 3; ++x) {
                                const int u = e1[x], q = e2[x];
                                sx[x] = s1[x][u][q];
                                double dd = 4.0 * ea * eb * s1[x][u + 1][q + 1];
                                if (u > 0) dd -= 2.0 * eb * u * s1[x][u - 1][q + 1];
                                if (q > 0) dd -= 2.0 * ea * q * s1[x][u + 1][q - 1];
                                if (u > 0 && q > 0) dd += (double)u * q * s1[x][u - 1][q - 1];
                                tx[x] = 0.5 * dd;
                            }
                            s[(size_t)i * nbb + j] += w * pre * sx[0] * sx[1] * sx[2];
                            t[(size_t)i * nbb + j] += w * pre * (tx[0] * sx[1] * sx[2] + sx[0] * tx[1] * sx[2] +
                                                                 sx[0] * sx[1] * tx[2]);
                            v[(size_t)i * nbb + j] += w * vv[(size_t)i * nbb + j];
                        }
                }
            std::vector<double> fs, ft, fv;
            to_functions(ta, tb, s, na, nbb, fs);
            to_functions(ta, tb, t, na, nbb, ft);
            to_functions(ta, tb, v, na, nbb, fv);
            const int nfa = nfunc_of(ta), nfb = nfunc_of(tb);
            const int oa = B->aosh[a], ob = B->aosh[b];
            for (int i = 0; i < nfa; ++i)
                for (int j = 0; j < nfb; ++j) {
                    const size_t k1 = (size_t)(oa + i) * nb + (ob + j), k2 = (size_t)(ob + j) * nb + (oa + i);
                    if (S) S[k1] = S[k2] = fs[(size_t)i * nfb + j];
                    if (T) T[k1] = T[k2] = ft[(size_t)i * nfb + j];
                    if (V) V[k1] = V[k2] = fv[(size_t)i * nfb + j];
                }
        }
    return HFGPU_OK;
}

// ------------------------------------------------------------- device ----
// The same integrals on the GPU: one thread per shell pair (a >= b), pairs
// sorted by shell-type class so that a warp walks one recursion plan.  The
// nuclear-attraction plan of each class (the NucPlan ops above, built once
// on the host) is read from global memory by the whole warp.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

namespace {

constexpr int ONEE_MAXOPS = 384;   // largest plan: (d|d), checked on the host
constexpr int ONEE_MAXC = 6;       // Cartesian components per shell

struct OneeClass {
    int op0, nops, tg0;            // plan slice and its (i, j) targets
    int na, nbc, la, lb;           // Cartesian counts and angular momenta
    int ta, tb;                    // shell types
    int ca[ONEE_MAXC][3], cb[ONEE_MAXC][3];
    int sa[ONEE_MAXC], sb[ONEE_MAXC];  // component belongs to an L shell's p part
};

struct OneeArgs {
    const int2* pairs;             // (a, b) shell indices, a >= b
    const int* pcls;               // class of each pair
    int npairs;
    const OneeClass* cls;
    const NucOp* ops;
    const int* targets;
    const int* shtyp;
    const int* nzet;
    const int* aosh;
    const double* xsh;
    const double* zeta;
    const double* djk;
    const double* djkl;
    int maxprim, nb, natom;
    const double* charges;
    const double* xyz;
    double* S;
    double* T;
    double* V;
};

__device__ void to_functions_dev(int ta, int tb, const double* cart, int nca, int ncb, double* out) {
    const double r3 = 1.7320508075688772935;
    const double H[5][6] = {{-.5, 0, 0, -.5, 0, 1.0}, {0, 0, r3, 0, 0, 0}, {0, 0, 0, 0, r3, 0},
                            {0, r3, 0, 0, 0, 0}, {r3 / 2, 0, 0, -r3 / 2, 0, 0}};
    double tmp[5 * ONEE_MAXC];
    const int nfa = ta == HFGPU_SHELL_D ? 5 : nca, nfb = tb == HFGPU_SHELL_D ? 5 : ncb;
    for (int j = 0; j < ncb; ++j)
        for (int i = 0; i < nfa; ++i) {
            double v = 0.0;
            if (ta == HFGPU_SHELL_D)
                for (int c = 0; c < 6; ++c) v += H[i][c] * cart[c * ncb + j];
            else
                v = cart[i * ncb + j];
            tmp[i * ncb + j] = v;
        }
    for (int i = 0; i < nfa; ++i)
        for (int j = 0; j < nfb; ++j) {
            double v = 0.0;
            if (tb == HFGPU_SHELL_D)
                for (int c = 0; c < 6; ++c) v += H[j][c] * tmp[i * ncb + c];
            else
                v = tmp[i * ncb + j];
            out[i * nfb + j] = v;
        }
}

__global__ void __launch_bounds__(128) k_onee(OneeArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.npairs) return;
    const int2 pr = a.pairs[t];
    const OneeClass& C = a.cls[a.pcls[t]];
    const int sa = pr.x, sb = pr.y, na = C.na, nbc = C.nbc, MP = a.maxprim;
    double s[ONEE_MAXC * ONEE_MAXC] = {}, tk[ONEE_MAXC * ONEE_MAXC] = {}, v[ONEE_MAXC * ONEE_MAXC] = {};
    double work[ONEE_MAXOPS];
    const double* A = a.xsh + 3 * sa;
    const double* B = a.xsh + 3 * sb;
    double AB2 = 0.0;
    for (int x = 0; x < 3; ++x) AB2 += (A[x] - B[x]) * (A[x] - B[x]);
    for (int za = 0; za < a.nzet[sa]; ++za)
        for (int zb = 0; zb < a.nzet[sb]; ++zb) {
            const double ea = a.zeta[(size_t)sa * MP + za], eb = a.zeta[(size_t)sb * MP + zb];
            const double p = ea + eb, mu = ea * eb / p;
            double P[3], PA[3], PB[3];
            for (int x = 0; x < 3; ++x) {
                P[x] = (ea * A[x] + eb * B[x]) / p;
                PA[x] = P[x] - A[x];
                PB[x] = P[x] - B[x];
            }
            const double K = exp(-mu * AB2);
            const double da = a.djk[(size_t)sa * MP + za], db = a.djk[(size_t)sb * MP + zb];
            const double ra = C.ta == HFGPU_SHELL_L ? a.djkl[(size_t)sa * MP + za] : 1.0;
            const double rb = C.tb == HFGPU_SHELL_L ? a.djkl[(size_t)sb * MP + zb] : 1.0;
            double s1[3][5][5];
            for (int x = 0; x < 3; ++x) overlap_1d(PA[x], PB[x], p, C.la + 1, C.lb + 1, s1[x]);
            const double pre = pow(PI_D / p, 1.5) * K;
            double vv[ONEE_MAXC * ONEE_MAXC] = {};
            const int L = C.la + C.lb;
            for (int c = 0; c < a.natom; ++c) {
                double PC[3], PC2 = 0.0, Fm[16], base[16];
                for (int x = 0; x < 3; ++x) {
                    PC[x] = P[x] - a.xyz[3 * c + x];
                    PC2 += PC[x] * PC[x];
                }
                boys_acc(L, p * PC2, Fm);
                for (int m = 0; m <= L; ++m) base[m] = 2.0 * PI_D / p * K * Fm[m];
                const double h = 0.5 / p;
                for (int o = 0; o < C.nops; ++o) {
                    const NucOp op = a.ops[C.op0 + o];
                    double x;
                    if (op.kind == 0) {
                        x = base[op.m];
                    } else {
                        const double g = op.kind == 1 ? PA[op.ax] : PB[op.ax];
                        x = g * work[op.c0] - PC[op.ax] * work[op.c1];
                        if (op.n1) x += h * op.n1 * (work[op.c2] - work[op.c3]);
                        if (op.n2) x += h * op.n2 * (work[op.c4] - work[op.c5]);
                    }
                    work[o] = x;
                }
                for (int q = 0; q < na * nbc; ++q) vv[q] -= a.charges[c] * work[a.targets[C.tg0 + q]];
            }
            for (int i = 0; i < na; ++i)
                for (int j = 0; j < nbc; ++j) {
                    const double w = da * db * (C.sa[i] ? ra : 1.0) * (C.sb[j] ? rb : 1.0);
                    double sx[3], tx[3];
                    for (int x = 0; x < 3; ++x) {
                        const int u = C.ca[i][x], q = C.cb[j][x];
                        sx[x] = s1[x][u][q];
                        double dd = 4.0 * ea * eb * s1[x][u + 1][q + 1];
                        if (u > 0) dd -= 2.0 * eb * u * s1[x][u - 1][q + 1];
                        if (q > 0) dd -= 2.0 * ea * q * s1[x][u + 1][q - 1];
                        if (u > 0 && q > 0) dd += (double)u * q * s1[x][u - 1][q - 1];
                        tx[x] = 0.5 * dd;
                    }
                    s[i * nbc + j] += w * pre * sx[0] * sx[1] * sx[2];
                    tk[i * nbc + j] += w * pre * (tx[0] * sx[1] * sx[2] + sx[0] * tx[1] * sx[2] + sx[0] * sx[1] * tx[2]);
                    v[i * nbc + j] += w * vv[i * nbc + j];
                }
        }
    double f[25];
    const int nfa = C.ta == HFGPU_SHELL_D ? 5 : na, nfb = C.tb == HFGPU_SHELL_D ? 5 : nbc;
    const int oa = a.aosh[sa], ob = a.aosh[sb], nb = a.nb;
    double* outs[3] = {a.S, a.T, a.V};
    const double* ins[3] = {s, tk, v};
    for (int w = 0; w < 3; ++w) {
        if (!outs[w]) continue;
        to_functions_dev(C.ta, C.tb, ins[w], na, nbc, f);
        for (int i = 0; i < nfa; ++i)
            for (int j = 0; j < nfb; ++j) {
                outs[w][(size_t)(oa + i) * nb + (ob + j)] = f[i * nfb + j];
                outs[w][(size_t)(ob + j) * nb + (oa + i)] = f[i * nfb + j];
            }
    }
}

thread_local std::string g_onee_err;

}  // namespace

#include <mutex>

namespace hfgpu {
void set_last_error(const std::string& msg);  // hfgpu.cu
cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t st);  // hfgpu.cu: the library's memory pool
}

namespace {
// Stream-ordered allocation and upload on the call's own stream: no
// device-wide synchronisation, so calls of concurrent jobs (and a capture in
// another thread) go on undisturbed.  Pageable sources are staged by the
// copy before it returns.
template <typename T>
cudaError_t up(T** d, const std::vector<T>& h, cudaStream_t st) {
    cudaError_t e = hfgpu::pool_alloc((void**)d, std::max<size_t>(h.size(), 1) * sizeof(T), st);
    if (e == cudaSuccess && !h.empty())
        e = cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st);
    return e;
}
}  // namespace

extern "C" int hfgpu_one_electron_gpu(const hfgpu_basis* B, int natom, const double* charges, const double* xyz,
                                      double* S, double* T, double* V) {
    if (!B || B->nsh <= 0 || B->nb <= 0 || natom <= 0 || !charges || !xyz) {
        hfgpu::set_last_error("hfgpu_one_electron_gpu: bad arguments");
        return HFGPU_ERR_ARG;
    }
    const int nb = B->nb, nsh = B->nsh, MP = B->maxprim;
    // one recursion plan per pair of shell types
    std::map<std::pair<int, int>, int> clsid;
    std::vector<OneeClass> cls;
    std::vector<NucOp> ops;
    std::vector<int> targets;
    std::vector<int2> pairs;
    std::vector<int> pcls;
    std::vector<C3> ca, cb;
    std::vector<int> ia, ib;
    for (int a = 0; a < nsh; ++a)
        for (int b = 0; b <= a; ++b) {
            const int ta = B->shtyp[a], tb = B->shtyp[b];
            auto key = std::make_pair(ta, tb);
            auto it = clsid.find(key);
            if (it == clsid.end()) {
                carts_of(ta, ca, ia);
                carts_of(tb, cb, ib);
                OneeClass c{};
                c.na = (int)ca.size();
                c.nbc = (int)cb.size();
                c.la = ta == HFGPU_SHELL_D ? 2 : ta == HFGPU_SHELL_S ? 0 : 1;
                c.lb = tb == HFGPU_SHELL_D ? 2 : tb == HFGPU_SHELL_S ? 0 : 1;
                c.ta = ta;
                c.tb = tb;
                for (int i = 0; i < c.na; ++i) {
                    c.ca[i][0] = ca[i].x; c.ca[i][1] = ca[i].y; c.ca[i][2] = ca[i].z;
                    c.sa[i] = ia[i];
                }
                for (int j = 0; j < c.nbc; ++j) {
                    c.cb[j][0] = cb[j].x; c.cb[j][1] = cb[j].y; c.cb[j][2] = cb[j].z;
                    c.sb[j] = ib[j];
                }
                NucPlan plan;
                std::vector<int> tg;
                for (int i = 0; i < c.na; ++i)
                    for (int j = 0; j < c.nbc; ++j) {
                        int ai[3] = {ca[i].x, ca[i].y, ca[i].z}, bj[3] = {cb[j].x, cb[j].y, cb[j].z};
                        tg.push_back(plan.get(ai, bj, 0));
                    }
                if ((int)plan.ops.size() > ONEE_MAXOPS) {
                    hfgpu::set_last_error("hfgpu_one_electron_gpu: recursion plan larger than the kernel's buffer");
                    return HFGPU_ERR_UNSUPPORTED;
                }
                c.op0 = (int)ops.size();
                c.nops = (int)plan.ops.size();
                c.tg0 = (int)targets.size();
                ops.insert(ops.end(), plan.ops.begin(), plan.ops.end());
                targets.insert(targets.end(), tg.begin(), tg.end());
                it = clsid.emplace(key, (int)cls.size()).first;
                cls.push_back(c);
            }
            pairs.push_back(make_int2(a, b));
            pcls.push_back(it->second);
        }
    // pairs of one class next to each other: a warp walks one plan
    std::vector<int> ord(pairs.size());
    for (size_t i = 0; i < ord.size(); ++i) ord[i] = (int)i;
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return pcls[x] < pcls[y]; });
    std::vector<int2> sp(pairs.size());
    std::vector<int> sc(pairs.size());
    for (size_t i = 0; i < ord.size(); ++i) {
        sp[i] = pairs[ord[i]];
        sc[i] = pcls[ord[i]];
    }
    std::vector<int> shtyp(B->shtyp, B->shtyp + nsh), nzet(B->nzet, B->nzet + nsh), aosh(B->aosh, B->aosh + nsh);
    std::vector<double> xsh(B->xsh, B->xsh + 3 * nsh), zeta(B->zeta, B->zeta + (size_t)nsh * MP);
    std::vector<double> djk(B->djk, B->djk + (size_t)nsh * MP), djkl(B->djkl, B->djkl + (size_t)nsh * MP);
    std::vector<double> ch(charges, charges + natom), xz(xyz, xyz + 3 * natom);
    OneeArgs g{};
    int2* d_pairs = nullptr;
    int *d_pcls = nullptr, *d_targets = nullptr, *d_shtyp = nullptr, *d_nzet = nullptr, *d_aosh = nullptr;
    OneeClass* d_cls = nullptr;
    NucOp* d_ops = nullptr;
    double *d_xsh = nullptr, *d_zeta = nullptr, *d_djk = nullptr, *d_djkl = nullptr, *d_ch = nullptr,
           *d_xyz = nullptr, *d_out = nullptr;
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        hfgpu::set_last_error(std::string("hfgpu_one_electron_gpu: ") + cudaGetErrorString(e));
        return HFGPU_ERR_CUDA;
    }
    e = up(&d_pairs, sp, st);
    if (e == cudaSuccess) e = up(&d_pcls, sc, st);
    if (e == cudaSuccess) e = up(&d_cls, cls, st);
    if (e == cudaSuccess) e = up(&d_ops, ops, st);
    if (e == cudaSuccess) e = up(&d_targets, targets, st);
    if (e == cudaSuccess) e = up(&d_shtyp, shtyp, st);
    if (e == cudaSuccess) e = up(&d_nzet, nzet, st);
    if (e == cudaSuccess) e = up(&d_aosh, aosh, st);
    if (e == cudaSuccess) e = up(&d_xsh, xsh, st);
    if (e == cudaSuccess) e = up(&d_zeta, zeta, st);
    if (e == cudaSuccess) e = up(&d_djk, djk, st);
    if (e == cudaSuccess) e = up(&d_djkl, djkl, st);
    if (e == cudaSuccess) e = up(&d_ch, ch, st);
    if (e == cudaSuccess) e = up(&d_xyz, xz, st);
    const size_t nb2 = (size_t)nb * nb;
    if (e == cudaSuccess) e = hfgpu::pool_alloc((void**)&d_out, 3 * nb2 * sizeof(double), st);
    if (e == cudaSuccess) {
        g.pairs = d_pairs; g.pcls = d_pcls; g.npairs = (int)sp.size(); g.cls = d_cls; g.ops = d_ops;
        g.targets = d_targets; g.shtyp = d_shtyp; g.nzet = d_nzet; g.aosh = d_aosh; g.xsh = d_xsh;
        g.zeta = d_zeta; g.djk = d_djk; g.djkl = d_djkl; g.maxprim = MP; g.nb = nb; g.natom = natom;
        g.charges = d_ch; g.xyz = d_xyz;
        g.S = S ? d_out : nullptr;
        g.T = T ? d_out + nb2 : nullptr;
        g.V = V ? d_out + 2 * nb2 : nullptr;
        k_onee<<<(g.npairs + 127) / 128, 128, 0, st>>>(g);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && S) e = cudaMemcpyAsync(S, d_out, nb2 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && T)
        e = cudaMemcpyAsync(T, d_out + nb2, nb2 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && V)
        e = cudaMemcpyAsync(V, d_out + 2 * nb2, nb2 * sizeof(double), cudaMemcpyDeviceToHost, st);
    void* bufs[] = {d_pairs, d_pcls, d_cls, d_ops, d_targets, d_shtyp, d_nzet, d_aosh, d_xsh, d_zeta, d_djk,
                    d_djkl, d_ch, d_xyz, d_out};
    for (void* b : bufs)
        if (b) cudaFreeAsync(b, st);
    const cudaError_t es = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = es;
    cudaStreamDestroy(st);
    if (e != cudaSuccess) {
        hfgpu::set_last_error(std::string("hfgpu_one_electron_gpu: ") + cudaGetErrorString(e));
        return HFGPU_ERR_CUDA;
    }
    return HFGPU_OK;
}
