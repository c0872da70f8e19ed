// Host-compiled check of the generated class code (test infrastructure).
//
// The CUDA device functions that evaluate contracted ERI blocks and scatter
// them into the Fock buffer are plain arithmetic; compiled here for the CPU
// with a few shims, they can be compared against the CPU oracle without a
// GPU.  Only tests/test_generated_host.py builds and loads this file.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#define __device__
#define __host__
#define __forceinline__ inline
static inline int __double2int_rn(double x) { return (int)std::nearbyint(x); }
static inline int __float2int_rn(float x) { return (int)std::nearbyintf(x); }
#define __expf(x) std::exp((float)(x))
static inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }
static inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }
template <class T>
static inline T __ldg(const T* p) { return *p; }
static inline double atomicAdd(double* p, double v) {
    double o = *p;
    *p += v;
    return o;
}

#include "types.cuh"
#include "pairs.hpp"
#include "generated/all_classes.inc"

using namespace hfgpu;

struct HC {
    const hfgpu_basis* B;
    std::vector<double> bt;
    std::vector<float> btf;
};

template <int M>
static void boys_m(const double* bt, double T, double* out) {
    boys_eval<M>(T, bt + (size_t)M * BOYS_BLK, out);
}

extern "C" {

// F_0..F_M(T) from the device Boys evaluation (table, Taylor, downward
// recursion with the tabulated exponential), compiled for the host
void hc_boys(const void* hv, int M, double T, double* out) {
    const double* bt = ((const HC*)hv)->bt.data();
    switch (M) {
        case 0: boys_m<0>(bt, T, out); break;
        case 1: boys_m<1>(bt, T, out); break;
        case 2: boys_m<2>(bt, T, out); break;
        case 3: boys_m<3>(bt, T, out); break;
        case 4: boys_m<4>(bt, T, out); break;
        case 5: boys_m<5>(bt, T, out); break;
        case 6: boys_m<6>(bt, T, out); break;
        case 7: boys_m<7>(bt, T, out); break;
        default: boys_m<8>(bt, T, out); break;
    }
}

void* hc_create(const hfgpu_basis* B) {
    HC* h = new HC();
    h->B = B;
    build_boys_table(h->bt, h->btf);
    return h;
}

void hc_destroy(void* h) { delete (HC*)h; }

// ERI block of class cls for the GPU-oriented pairs (a,b) and (c,d).
int hc_eri(void* hh, int cls, int L, int a, int b, int c, int d, int f32, double* out) {
    HC* h = (HC*)hh;
    std::vector<GPrim> prims;
    GPair bra = make_pair(h->B, a, b, prims);
    GPair ket = make_pair(h->B, c, d, prims);
    std::vector<double> soa = prims_soa(prims);
    const PrimSoA ps = soa_view(soa.data(), prims.size());
    const double* t = h->bt.data() + (size_t)L * BOYS_BLK;
    const float* tf = h->btf.data() + (size_t)L * BOYS_BLK;
    HOST_ERI[cls](bra, ket, ps, t, tf, out, f32);
    return 0;
}

// Role scatter of a full ERI block (returns 1 for single-function classes).
int hc_scatter(void* hh, int cls, int a, int b, int c, int d, const double* e, double s, const double* P,
               double* G, int nb, int jonly) {
    HC* h = (HC*)hh;
    std::vector<GPrim> prims;
    GPair bra = make_pair(h->B, a, b, prims);
    GPair ket = make_pair(h->B, c, d, prims);
    return HOST_SCAT[cls](e, s, bra, ket, P, G, nb, jonly != 0);
}

}
