/*
 * bcpnn_device.cuh -- sm_100a kernels of the plain FP32 ProcUpdLazy path.
 *
 * Compiled with -fmad=false: every float expression below is evaluated with
 * the same IEEE operations, in the same order, as gsbn's CPU path
 * (src/gsbn/procedures/ProcUpdLazy/Pop.cpp, Proj.cpp), so the results are
 * bit-identical to a CPU replay that uses the same exp/log definitions
 * (include/bcpnn_numerics.h).
 *
 * Execution model (one network, one GPU):
 *   - tick_kernel: one CTA per (population, destination HCU).  A tick of gsbn
 *     touches, for destination HCU h, only state that belongs to h (its MCUs,
 *     its slots, its cells), except the delayed presynaptic spikes read by the
 *     delay queue, which come from the previous tick.  So one CTA does, for HCU
 *     h: support/softmax/spike sampling (Pop.cpp:229-323), the j-trace step of
 *     every incoming projection (Proj.cpp:310-363), the row updates of h's
 *     active rows with ordered epsc accumulation (Proj.cpp:365-479, 667-720),
 *     the column updates of h's spiking MCUs (Proj.cpp:481-536, 722-760) and
 *     the delay queue of h's slots with ascending warp-ballot compaction of
 *     the next tick's active rows (Proj.cpp:621-664).  The kernel boundary is
 *     the only grid-wide synchronisation per tick.
 *   - Values read across CTAs inside a tick (the population's MCU-0 support
 *     that seeds every HCU's softmax max, Pop.cpp:270; si) are double
 *     buffered by tick parity: a tick reads buffer prev and writes buffer cur.
 *   - all_rows_kernel / all_cells_kernel: the all-cells catch-up at a change
 *     of prn (Proj.cpp:209-308, 538-588), a streaming pass over every row and
 *     every cell.
 *   - The closed-form decay factors depend on the elapsed ticks pdt only; they
 *     are tabulated per projection and per kp by build_table_kernel with the
 *     same float expressions the reference evaluates inline, so a table
 *     lookup returns the very bits an inline evaluation would.
 */
#ifndef BCPNN_DEVICE_CUH
#define BCPNN_DEVICE_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "bcpnn_numerics.h"

namespace bcpnn {

constexpr int kBlock = 512;         /* threads of the block-wide helpers below; the
                                       tick kernel defines its own CTA size  */
constexpr int kWarps = kBlock / 32;
constexpr int kMaxPops = 4096;      /* populations per network (batches of networks) */
constexpr int kMaxProj = 4096;      /* projections per network                 */
constexpr int kRowChunkCells = kBlock; /* row cells staged per chunk (one per thread) */
constexpr int kColU = 2;            /* column cells per thread per batch         */
constexpr int kColUnit = 256;       /* slots of one column work unit (see NetDev::col_ring) */
constexpr int kMaxIn = 8;           /* incoming projections per population       */

/* error bits of NetDev::err */
constexpr int kErrIndex = 1;        /* ii out of the source population range   */
constexpr int kErrBarrier = 2;      /* a grid barrier wait ran out of time      */
constexpr int kErrColumns = 4;      /* a wait for deferred column work ran out of time */
constexpr int kErrSeed = 8;         /* a published softmax seed carried the wrong tick tag */

/* Phase probe of the tick kernel (compile-time flag BCPNN_PHASE_PROBE, off in
   the default build): per CTA, the SM clock cycles spent in each phase of a
   tick, summed over ticks.  Group A's first thread records slots 0-15, group
   B's first thread slots 16-30; slot kProbeTicks counts the ticks. */
constexpr int kProbeSlots = 32;
constexpr int kProbeTicks = 31;
constexpr int kProbeCtas = 4096;
#ifdef BCPNN_PHASE_PROBE
__device__ unsigned long long g_phase_probe[kProbeCtas * kProbeSlots];
/* the CTA's counters during a launch: shared memory, so that a mark costs a
   clock read and a shared-memory add, not a global round trip */
__shared__ unsigned long long g_probe_smem[kProbeSlots];
#endif

struct PopDev {
  int H, M, n, hcu_start, mcu_start, dim_proj, id;
  uint32_t rng_seed, rng_pop; /* Philox key of this population's streams: (rng_seed, rng_pop*16 + stream) */
  float taumdt, wtagain, maxfqdt, igain, wgain, lgbias, snoise;
  float* dsup[2];   /* [n], by tick parity                                  */
  float* act;       /* [n]                                                  */
  float* epsc[2];   /* [dim_proj][n], by tick parity                        */
  float* bj[2];     /* [dim_proj][n], by tick parity                        */
  int8_t* spike;    /* [n] spikes of the last tick (spike_<pop>)            */
  int* counter;     /* [n] .counter_<pop>                                   */
  uint32_t* spk_log;/* [max_ticks][log_words]                               */
  int log_words;
  int n_in;         /* projections whose destination is this population    */
  const int* in_proj;
  int n_out;        /* projections whose si this population feeds          */
  const int* out_proj;
  int ext;          /* external spike replay                                */
  const int* ext_off; /* [ext_t1 - ext_t0 + 1] offsets by simstep - ext_t0 */
  const int* ext_idx;
  int ext_t0, ext_t1;
  /* ProcUpdMulti only */
  float* ada;        /* [n] adaptation current                                */
  int8_t* ring;      /* [ring_len][n] spikes by simstep % ring_len          */
  int ring_len;      /* "spike buffer size"                                  */
  float tauadt, adgain;
};

struct ProjDev {
  int src, dest, H, M, C, Ns, proj_in_pop;
  int fp64;                             /* decay tables: 0 gsbn's closed form, 1 FP64-built propagators */
  float taupdt, ke, kzi, kzj, kepsc, kfti, kftj, eps, eps2, wgain, bgain;
  int* ii; int* di; int* qi;            /* [H*C] */
  float* pi; float* ei; float* zi;      /* [H*C] */
  int* ti;                              /* [H*C] */
  float* pj; float* ej; float* zj;      /* [H*M] */
  float4* cell;                         /* [H*C*M] (pij, eij, zi2, zj2) */
  int* tij;                             /* [H*C*M] */
  float* wij;                           /* [H*C*M] */
  int8_t* si[2];                        /* [Ns], by tick parity */
  int* list;                            /* [H*C] active rows, per HCU segment */
  int* list_cnt;                        /* [H] */
};

struct NetDev {
  int n_pops, n_projs;
  float dt, poisson_hz;
  uint32_t seed;
  const PopDev* pops;   /* [n_pops], device array  */
  const ProjDev* projs; /* [n_projs], device array */
  const int* cta_pop;   /* CTA -> population */
  const int* cta_hcu;   /* CTA -> HCU        */
  float* lginp;         /* [total MCUs] host-set stimulus */
  float* wmask;         /* [total HCUs] */
  uint32_t* ss_log;     /* [max_ticks][n_projs] debug flags of ProcSpkRec */
  unsigned long long* counters; /* row cells, col cells, all cells */
  int* err;
  /* Deferred column work of the persistent launch.  The column updates of the
     MCUs that spike in tick t are done in tick t+1 by every CTA of the grid
     instead of by the spiking HCU's CTA alone.  A unit is up to kColUnit slots
     of one spiking column: (owner CTA, projection, first row h*C + part*kColUnit,
     MCU | rows << 16).  Two ring halves by tick parity, col_cap units each. */
  int4* col_ring;
  int col_cap;
  /* [n_pops][2] the softmax seed of the next tick (dsup of the population's
     MCU 0, Pop.cpp:270), published by the population's HCU-0 CTA at the end
     of a tick of the persistent launch, before its barrier arrival: (tick
     tag << 32) | float bits, in slot [tag & 1].  The other CTAs' barrier
     threads load it while they poll, so it costs no round trip after the
     barrier; the tag (RunParams::serial0 + tick) certifies it.  Two slots:
     the publisher can be a tick ahead of a reader that has not yet seen the
     barrier complete (it publishes tick t+1's seed before every CTA has read
     tick t's), never two. */
  unsigned long long* seed64;
};

/* Decay table entry for one elapsed-tick count d: four float4
   [0] cell: Ep, Epe, Epzz, Ep*D3
   [1] cell: Ee, (Ezi*Ezj)*D3, Emzi, Emzj
   [2] row:  Ep, Epe, Epzi, Ep*(ke-kzi)
   [3] row:  Ee, Eezi, Ee*(ke-kzi), Emzi
   with a = kp*d, b = ke*d, c = kzi*d, e = kzj*d (float products),
   Ep = exp(a), Epe = exp(a-b), Epzz = exp((a-c)-e), Ee = exp(b),
   Ezi = exp(c), Ezj = exp(e), Emzi = exp(-kzi*d), Emzj = exp(-kzj*d),
   Epzi = exp(a-c), Eezi = exp(b-c), D3 = (kzi-ke)+kzj.                     */
struct RunParams {
  int simstep0;   /* simstep of the first tick of the run */
  int k0;         /* ticks executed before the run (parity base) */
  int n_ticks;
  float prn, old_prn;
  const float* lginp;   /* stimulus of the run: [total MCUs] */
  const float* wmask;   /* [total HCUs] */
  const struct TabRef* tabs;  /* [n_projs] decay tables of the run */
  unsigned int serial0; /* tag of the run's first tick (never repeats between consecutive ticks, see seed64) */
};

/* constants of the closed form for one kp */
struct Coef {
  float kp, ke, kzi, kzj, kekp, Dekp, Dpzi, Dezi, D2, D3;
  int fp64; /* tables hold FP64-built propagator coefficients (see fp64_entry) */
};

__host__ __device__ __forceinline__ Coef make_coef(float kp, float ke, float kzi, float kzj, int fp64 = 0) {
  Coef k;
  k.fp64 = fp64;
  k.kp = kp; k.ke = ke; k.kzi = kzi; k.kzj = kzj;
  k.kekp = ke * kp;
  k.Dekp = ke - kp;
  k.Dpzi = kp - kzi;
  k.Dezi = ke - kzi;
  k.D2 = (kzi - kp) + kzj;
  k.D3 = (kzi - ke) + kzj;
  return k;
}

/* reciprocals (double, correctly rounded) of the closed form's constant
   divisors for one kp: 1/(ke-kp), 1/((kzi-kp)+kzj), 1/((kzi-ke)+kzj),
   1/(kp-kzi), 1/(ke-kzi), with the divisors evaluated in float as gsbn does */
struct RCoef {
  double Dekp, D2, D3, Dpzi, Dezi;
};

/* decay tables of one projection for a run */
struct TabRef {
  const float4* tab;      /* kp = taupdt*prn     */
  const float4* tab_old;  /* kp = taupdt*old_prn */
  const double2* rtab;    /* kp = taupdt*prn: reciprocals of the divisor entries, see build_table_kernel */
  int len, old_len;
  Coef k;                 /* kp = taupdt*prn */
  RCoef rk;               /* kp = taupdt*prn */
};


/* The transcendental functions are real calls in device code: several call
   sites share one copy of their instructions, which keeps the tick kernel's
   instruction footprint small (its rarely taken paths are otherwise fetched
   from L2 every tick). */
__device__ __noinline__ float dev_expf(float x) { return bx_expf(x); }
__device__ __noinline__ float dev_logf(float x) { return bx_logf(x); }
__device__ __noinline__ float dev_normal01(uint32_t seed, uint32_t pop, uint32_t tick, uint32_t mcu) {
  return bx_normal01(seed, pop, tick, mcu);
}

/* table entry computed inline (used to build tables and for an elapsed time
   beyond the table) */
__device__ __forceinline__ void table_entry(float kp, float ke, float kzi, float kzj, int d, float4& o0, float4& o1,
                                            float4& o2, float4& o3) {
  float fd = (float)d;
  float a = kp * fd, b = ke * fd, c = kzi * fd, e = kzj * fd;
  float D3 = (kzi - ke) + kzj;
  float Dezi = ke - kzi;
  float Ep = dev_expf(a);
  float Epe = dev_expf(a - b);
  float Epzz = dev_expf((a - c) - e);
  float Ee = dev_expf(b);
  float Ezi = dev_expf(c);
  float Ezj = dev_expf(e);
  float Emzi = dev_expf(-kzi * fd);
  float Emzj = dev_expf(-kzj * fd);
  float Epzi = dev_expf(a - c);
  float Eezi = dev_expf(b - c);
  o0 = make_float4(Ep, Epe, Epzz, Ep * D3);
  o1 = make_float4(Ee, (Ezi * Ezj) * D3, Emzi, Emzj);
  o2 = make_float4(Ep, Epe, Epzi, Ep * Dezi);
  o3 = make_float4(Ee, Eezi, Ee * Dezi, Emzi);
}

/* FP64-built propagator of the trace chain over d ticks.  Between events
   the traces obey linear ODEs (rates per tick):
     cells: p' = kp (e - p), e' = ke (s - e), s' = -(kzi + kzj) s, s = zi2 zj2
     rows:  p' = kp (e - p), e' = ke (z - e), z' = -kzi z
   so x(d) = expm(d A) x(0) with A upper bidiagonal.  gsbn's closed form
   (Proj.cpp:435-443) is this solution written with divided differences
   1/(ke - kzi), 1/((kzi - ke) + kzj), ..., which cancel catastrophically when
   time constants nearly coincide.  expm(d A) by scaling and squaring with a
   Taylor series (Moler & Van Loan, "Nineteen dubious ways...", 1978/2003,
   method 3) uses products and sums only and does not care how close the
   rates are; it runs in double and is rounded once to float.
   entry[0] = (P<-p, P<-e, P<-s, E<-e)   entry[1] = (E<-s, e^{-kzi d}, e^{-kzj d}, 0)
   entry[2] = (P<-p, P<-e, P<-z, E<-e)   entry[3] = (E<-z, e^{-kzi d}, 0, 0)       */
__device__ __forceinline__ void expm3_upper(double a00, double a01, double a11, double a12, double a22, double d,
                                            double E[6]) {
  /* M = d A = [[m00, m01, 0], [0, m11, m12], [0, 0, m22]]; E = (E00, E01, E02, E11, E12, E22) */
  double m00 = a00 * d, m01 = a01 * d, m11 = a11 * d, m12 = a12 * d, m22 = a22 * d;
  double nrm = fmax(fabs(m00) + 0.0, fmax(fabs(m01) + fabs(m11), fabs(m12) + fabs(m22)));
  if (!(nrm <= 1.7976931348623157e308)) { /* an infinite or NaN rate: no propagator exists */
    const double qnan = __longlong_as_double(0x7ff8000000000000LL);
    for (int k = 0; k < 6; k++) E[k] = qnan;
    return;
  }
  /* a finite norm is below 2^1024, so at most 1027 halvings reach 1/8 */
  int sq = 0;
  for (; sq < 1100 && nrm > 0.125; sq++) nrm *= 0.5;
  const double sc = ldexp(1.0, -sq);
  m00 *= sc; m01 *= sc; m11 *= sc; m12 *= sc; m22 *= sc;
  /* Taylor sum of exp(M): term T_k = T_{k-1} M / k, upper triangular */
  double t00 = 1, t01 = 0, t02 = 0, t11 = 1, t12 = 0, t22 = 1;
  double e00 = 1, e01 = 0, e02 = 0, e11 = 1, e12 = 0, e22 = 1;
  for (int k = 1; k <= 16; k++) {
    const double inv = 1.0 / (double)k;
    const double n00 = t00 * m00 * inv;
    const double n01 = (t00 * m01 + t01 * m11) * inv;
    const double n02 = (t01 * m12 + t02 * m22) * inv;
    const double n11 = t11 * m11 * inv;
    const double n12 = (t11 * m12 + t12 * m22) * inv;
    const double n22 = t22 * m22 * inv;
    t00 = n00; t01 = n01; t02 = n02; t11 = n11; t12 = n12; t22 = n22;
    e00 += t00; e01 += t01; e02 += t02; e11 += t11; e12 += t12; e22 += t22;
  }
  for (int i = 0; i < sq; i++) {
    const double s00 = e00 * e00, s01 = e00 * e01 + e01 * e11, s02 = e00 * e02 + e01 * e12 + e02 * e22;
    const double s11 = e11 * e11, s12 = e11 * e12 + e12 * e22, s22 = e22 * e22;
    e00 = s00; e01 = s01; e02 = s02; e11 = s11; e12 = s12; e22 = s22;
  }
  E[0] = e00; E[1] = e01; E[2] = e02; E[3] = e11; E[4] = e12; E[5] = e22;
}

__device__ __forceinline__ void fp64_entry(float kp, float ke, float kzi, float kzj, int d, float4& o0, float4& o1,
                                           float4& o2, float4& o3) {
  const double p = kp, e = ke, zi = kzi, zj = kzj;
  double C[6], R[6], J[6];
  expm3_upper(-p, p, -e, e, -(zi + zj), (double)d, C);
  expm3_upper(-p, p, -e, e, -zi, (double)d, R);
  expm3_upper(0.0, 0.0, 0.0, 0.0, -zj, (double)d, J); /* J[5] = e^{-kzj d} */
  o0 = make_float4((float)C[0], (float)C[1], (float)C[2], (float)C[3]);
  o1 = make_float4((float)C[4], (float)R[5], (float)J[5], 0.0f);
  o2 = make_float4((float)R[0], (float)R[1], (float)R[2], (float)R[3]);
  o3 = make_float4((float)R[4], (float)R[5], 0.0f, 0.0f);
}

__global__ void build_table_fp64_kernel(float4* tab, int len, float kp, float ke, float kzi, float kzj) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < len; d += gridDim.x * blockDim.x) {
    float4 t0, t1, t2, t3;
    fp64_entry(kp, ke, kzi, kzj, d, t0, t1, t2, t3);
    tab[(size_t)d * 4 + 0] = t0;
    tab[(size_t)d * 4 + 1] = t1;
    tab[(size_t)d * 4 + 2] = t2;
    tab[(size_t)d * 4 + 3] = t3;
  }
}

/* the cell part (entry[0], entry[1]) of the decay factors for d elapsed
   ticks, computed with the same float expressions as table_entry */
__device__ __forceinline__ void cell_factors(float kp, float ke, float kzi, float kzj, int d, float4& A, float4& B) {
  float fd = (float)d;
  float a = kp * fd, b = ke * fd, c = kzi * fd, e = kzj * fd;
  float D3 = (kzi - ke) + kzj;
  float Ep = bx_expf(a);
  float Epe = bx_expf(a - b);
  float Epzz = bx_expf((a - c) - e);
  float Ee = bx_expf(b);
  float Ezi = bx_expf(c);
  float Ezj = bx_expf(e);
  float Emzi = bx_expf(-kzi * fd);
  float Emzj = bx_expf(-kzj * fd);
  A = make_float4(Ep, Epe, Epzz, Ep * D3);
  B = make_float4(Ee, (Ezi * Ezj) * D3, Emzi, Emzj);
}

/* the two float4 of part `part` (0: cell, 2: row) of an entry beyond the
   table, computed; one out-of-line copy */
struct F4x2 {
  float4 a, b;
};

__device__ __noinline__ F4x2 table_pair_nl(float kp, float ke, float kzi, float kzj, int d, int part) {
  float4 t0, t1, t2, t3;
  table_entry(kp, ke, kzi, kzj, d, t0, t1, t2, t3);
  F4x2 r;
  if (part == 0) {
    r.a = t0;
    r.b = t1;
  } else {
    r.a = t2;
    r.b = t3;
  }
  return r;
}

/* the same for FP64-built propagators; a function of its own, so that the
   closed-form path's call carries none of its double-precision registers */
__device__ __noinline__ F4x2 table_pair_fp64_nl(float kp, float ke, float kzi, float kzj, int d, int part) {
  float4 t0, t1, t2, t3;
  fp64_entry(kp, ke, kzi, kzj, d, t0, t1, t2, t3);
  F4x2 r;
  if (part == 0) {
    r.a = t0;
    r.b = t1;
  } else {
    r.a = t2;
    r.b = t3;
  }
  return r;
}

__device__ __forceinline__ void table_pair(float kp, float ke, float kzi, float kzj, int d, int part, float4& A,
                                           float4& B, int fp64 = 0) {
  F4x2 r = fp64 ? table_pair_fp64_nl(kp, ke, kzi, kzj, d, part) : table_pair_nl(kp, ke, kzi, kzj, d, part);
  A = r.a;
  B = r.b;
}

__device__ __forceinline__ void load_entry(const float4* tab, int len, const Coef& k, int d, int part,
                                           float4& A, float4& B) {
  if (d < len) {
    A = tab[(size_t)d * 4 + part];
    B = tab[(size_t)d * 4 + part + 1];
  } else {
    table_pair(k.kp, k.ke, k.kzi, k.kzj, d, part, A, B, k.fp64);
  }
}

/* IEEE quotient a / b, rounded to nearest even: bit-identical to `a / b`.
   CUDA's float division leaves its quick path for a zero numerator, an
   infinite divisor, subnormal operands and quotients near the ends of the
   exponent range, and a warp waits for any lane on that path; in the decay
   closed forms most divisions meet one of these (traces that decayed to zero,
   exp() table entries that overflowed or underflowed).  So:
   - a zero numerator over a finite nonzero divisor, and a finite numerator
     over an infinite divisor, give their exact signed zero by selection;
   - a warp whose other lanes all have normal operands with exponents less
     than 100 apart divides in float (the quick path of `/`);
   - otherwise the warp divides in double and rounds once to float.  For
     p-bit operands a quotient rounded to p' >= 2p + 2 bits and then to p bits
     is the correctly rounded p-bit quotient (Figueroa, "When is double
     rounding innocuous?", SIGNUM Newsletter 30(3), 1995); 53 >= 2*24 + 2, and
     float operands are far from double's range limits;
   - an infinite or NaN operand, or a zero divisor, goes through `/` itself. */
__device__ __forceinline__ float div_rn(float a, float b) {
  const uint32_t ua = __float_as_uint(a), ub = __float_as_uint(b);
  const uint32_t aa = ua << 1, bb = ub << 1; /* magnitude bits */
  const bool zsel = (aa == 0u && bb - 1u < 0xff000000u) || (bb == 0xff000000u && aa < 0xff000000u);
  const uint32_t ea = aa >> 24, eb = bb >> 24; /* biased exponents */
  const bool quick = (ea - 1u < 254u) && (eb - 1u < 254u) && (ea - eb + 100u < 200u);
  const float za = zsel ? 1.0f : a, zb = zsel ? 1.0f : b;
  float q;
  if (__all_sync(__activemask(), zsel || quick)) {
    q = za / zb;
  } else if (!zsel && (ea == 255u || eb == 255u || bb == 0u)) {
    q = a / b;
  } else {
    q = __double2float_rn(__ddiv_rn((double)za, (double)zb));
  }
  return zsel ? __uint_as_float((ua ^ ub) & 0x80000000u) : q;
}

/* Closed-form decay of one cell over pdt ticks, Proj.cpp:435-443 (row),
   :519-527 (column), :269-277 (all).  A = entry[0], B = entry[1]. */
__device__ __forceinline__ void cell_decay(float& pij, float& eij, float& zi2, float& zj2, const Coef& k,
                                           float4 A, float4 B) {
  if (k.fp64) { /* FP64-built propagator (fp64_entry) */
    const float s = zi2 * zj2;
    const float pn = (A.x * pij + A.y * eij) + A.z * s;
    const float en = A.w * eij + B.x * s;
    pij = pn;
    eij = en;
    zi2 = zi2 * B.y;
    zj2 = zj2 * B.z;
    return;
  }
  float U = (((eij * k.kp) * k.kzi - (eij * k.ke) * k.kp) + (eij * k.kp) * k.kzj) + (k.kekp * zi2) * zj2;
  float V = (k.kekp * zi2) * zj2;
  float pn = div_rn(pij + div_rn(div_rn(U, k.Dekp) - div_rn(V, k.D2), k.D3), A.x) -
             div_rn(div_rn(A.y * U, k.Dekp) - div_rn(V * A.z, k.D2), A.w);
  float W = (k.ke * zi2) * zj2;
  float en = div_rn(eij + div_rn(W, k.D3), B.x) - div_rn(W, B.y);
  pij = pn;
  eij = en;
  zi2 = zi2 * B.z;
  zj2 = zj2 * B.w;
}

/* Out-of-line copies for the tick kernel: one body of the closed forms
   shared by its call sites keeps the kernel's instruction footprint small
   (each phase runs once per tick, so its code is fetched again every tick). */
__device__ __noinline__ float4 cell_decay_nl(float4 c, const Coef k, float4 A, float4 B) {
  cell_decay(c.x, c.y, c.z, c.w, k, A, B);
  return c;
}

/* Closed-form decay of the row traces, Proj.cpp:409-415 (row), :241-247
   (all).  A = entry[2], B = entry[3]. */
__device__ __forceinline__ void row_decay(float& pi, float& ei, float& zi, const Coef& k, float4 A, float4 B) {
  if (k.fp64) {
    const float pn = (A.x * pi + A.y * ei) + A.z * zi;
    const float en = A.w * ei + B.x * zi;
    pi = pn;
    ei = en;
    zi = zi * B.y;
    return;
  }
  float X = ((ei * k.kp) * k.kzi - (ei * k.ke) * k.kp) + k.kekp * zi;
  float Y = k.kekp * zi;
  float pn = div_rn(pi - div_rn(div_rn(X, k.Dekp) + div_rn(Y, k.Dpzi), k.Dezi), A.x) +
             div_rn(div_rn(A.y * X, k.Dekp) + div_rn(Y * A.z, k.Dpzi), A.w);
  float KZ = k.ke * zi;
  float en = div_rn(ei - div_rn(KZ, k.Dezi), B.x) + div_rn(KZ * B.y, B.z);
  pi = pn;
  ei = en;
  zi = zi * B.w;
}

__device__ __noinline__ float4 row_decay_nl(float4 r, const Coef k, float4 A, float4 B) {
  row_decay(r.x, r.y, r.z, k, A, B);
  return r;
}

/* The closed forms with every division a / b evaluated as
   RN_float(RN_double(a * r)), r = RN_double(1/b) precomputed (RCoef for the
   constant divisors, the reciprocal table for the table entries).  This is
   the correctly rounded float quotient whenever that quotient is a normal
   float: |a*r - a/b| <= 2^-51.9 |a/b|, while a/b, with 24-bit a and b, is
   never exactly a float midpoint and lies at least 2^-49 |a/b| away from
   every midpoint (a - m*b is a nonzero multiple of ulp(m)/2 * ulp(b)), so
   both round to the same float.  Below 2^-126 the float grid is uniform
   (2^-149): there a/b can be exactly a midpoint, and is otherwise at least
   2^-174 away from one (a - m*b is a nonzero multiple of 2^-150 ulp(b)),
   while |a*r - a/b| < 2^-178.  So a result in that range whose scaled value
   a*r*2^150 lies within 2^-25 of an odd integer (a midpoint) is ambiguous:
   the lane sets `slow` and the caller recomputes the whole decay with div_rn;
   every other result is RN(a/b).  Zeros, infinities and NaNs come out as IEEE
   division gives them (0*r, a*0, a*inf).  No branch and no vote per
   division, so the ten divisions of a cell overlap (checked against `/` on
   the GPU on random, subnormal, extreme and near-midpoint pairs, see
   bcpnn_selftest_division). */
__device__ __forceinline__ float qmul(float a, double r, bool& slow) {
  const double qd = (double)a * r;
  const float q = __double2float_rn(qd);
  if (fabs(qd) < 0x1p-126) {
    const double t = qd * 0x1p150; /* exact: the subnormal grid in half-units */
    const double n = rint(t);
    slow |= (fabs(t - n) < 0x1p-25) && ((((long long)n) & 1) != 0);
  }
  return q;
}

/* cell: A = entry[0], B = entry[1], R0 = (1/A.x, 1/A.w), R1 = (1/B.x, 1/B.y) */
__device__ __forceinline__ bool cell_decay_fast(float4& c, const Coef& k, const RCoef& rk, float4 A, float4 B,
                                                double2 R0, double2 R1) {
  bool slow = false;
  const float pij = c.x, eij = c.y, zi2 = c.z, zj2 = c.w;
  const float U = (((eij * k.kp) * k.kzi - (eij * k.ke) * k.kp) + (eij * k.kp) * k.kzj) + (k.kekp * zi2) * zj2;
  const float V = (k.kekp * zi2) * zj2;
  const float pn = qmul(pij + qmul(qmul(U, rk.Dekp, slow) - qmul(V, rk.D2, slow), rk.D3, slow), R0.x, slow) -
                   qmul(qmul(A.y * U, rk.Dekp, slow) - qmul(V * A.z, rk.D2, slow), R0.y, slow);
  const float W = (k.ke * zi2) * zj2;
  const float en = qmul(eij + qmul(W, rk.D3, slow), R1.x, slow) - qmul(W, R1.y, slow);
  if (slow) return false;
  c = make_float4(pn, en, zi2 * B.z, zj2 * B.w);
  return true;
}

/* row: A = entry[2], B = entry[3], R0 = (1/A.x, 1/A.w), R1 = (1/B.x, 1/B.z) */
__device__ __forceinline__ bool row_decay_fast(float4& r, const Coef& k, const RCoef& rk, float4 A, float4 B,
                                               double2 R0, double2 R1) {
  bool slow = false;
  const float pi = r.x, ei = r.y, zi = r.z;
  const float X = ((ei * k.kp) * k.kzi - (ei * k.ke) * k.kp) + k.kekp * zi;
  const float Y = k.kekp * zi;
  const float pn = qmul(pi - qmul(qmul(X, rk.Dekp, slow) + qmul(Y, rk.Dpzi, slow), rk.Dezi, slow), R0.x, slow) +
                   qmul(qmul(A.y * X, rk.Dekp, slow) + qmul(Y * A.z, rk.Dpzi, slow), R0.y, slow);
  const float KZ = k.ke * zi;
  const float en = qmul(ei - qmul(KZ, rk.Dezi, slow), R1.x, slow) + qmul(KZ * B.y, R1.y, slow);
  if (slow) return false;
  r = make_float4(pn, en, zi * B.w, r.w);
  return true;
}

/* One decay of a cell (row) on the float closed-form path: the reciprocal
   form, falling back to div_rn for a lane whose quotient is ambiguous.  Out
   of line: one copy of each body for all call sites; the constants come from
   the run's TabRef (in shared memory where the caller has a copy), so the
   call passes one pointer instead of 21 words of constants. */
#ifdef BCPNN_PHASE_PROBE
/* decays taken by the reciprocal form / by the div_rn fallback, per CTA */
#define PROBE_DECAY(slow) atomicAdd(&g_phase_probe[blockIdx.x % kProbeCtas * kProbeSlots + ((slow) ? 14 : 15)], 1ull)
#else
#define PROBE_DECAY(slow) do {} while (0)
#endif

__device__ __noinline__ float4 cell_step_nl(float4 c, const TabRef* __restrict__ T, float4 A, float4 B, double2 R0,
                                            double2 R1) {
  const Coef k = T->k;
  const RCoef rk = T->rk;
  float4 f = c;
  if (!k.fp64 && cell_decay_fast(f, k, rk, A, B, R0, R1)) {
    PROBE_DECAY(false);
    return f;
  }
  PROBE_DECAY(true);
  cell_decay(c.x, c.y, c.z, c.w, k, A, B);
  return c;
}

__device__ __noinline__ float4 row_step_nl(float4 r, const TabRef* __restrict__ T, float4 A, float4 B, double2 R0,
                                           double2 R1) {
  const Coef k = T->k;
  const RCoef rk = T->rk;
  float4 f = r;
  if (!k.fp64 && row_decay_fast(f, k, rk, A, B, R0, R1)) {
    PROBE_DECAY(false);
    return f;
  }
  PROBE_DECAY(true);
  row_decay(r.x, r.y, r.z, k, A, B);
  return r;
}

/* ------------------------------------------------------------------------ */

/* rtab, beside tab: for every d four double2, the correctly rounded
   reciprocals of the float divisor entries
     [0] cell: 1/Ep, 1/(Ep*D3)      [1] cell: 1/Ee, 1/((Ezi*Ezj)*D3)
     [2] row:  1/Ep, 1/(Ep*Dezi)    [3] row:  1/Ee, 1/(Ee*Dezi)           */
__device__ __forceinline__ void recip_part(float4 A, float4 B, int part, double2& R0, double2& R1) {
  R0 = make_double2(__drcp_rn((double)A.x), __drcp_rn((double)A.w));
  R1 = make_double2(__drcp_rn((double)B.x), __drcp_rn((double)(part == 0 ? B.y : B.z)));
}

__global__ void build_table_kernel(float4* tab, double2* rtab, int len, float kp, float ke, float kzi, float kzj) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < len; d += gridDim.x * blockDim.x) {
    float4 t0, t1, t2, t3;
    table_entry(kp, ke, kzi, kzj, d, t0, t1, t2, t3);
    tab[(size_t)d * 4 + 0] = t0;
    tab[(size_t)d * 4 + 1] = t1;
    tab[(size_t)d * 4 + 2] = t2;
    tab[(size_t)d * 4 + 3] = t3;
    double2 r0, r1, r2, r3;
    recip_part(t0, t1, 0, r0, r1);
    recip_part(t2, t3, 2, r2, r3);
    rtab[(size_t)d * 4 + 0] = r0;
    rtab[(size_t)d * 4 + 1] = r1;
    rtab[(size_t)d * 4 + 2] = r2;
    rtab[(size_t)d * 4 + 3] = r3;
  }
}

/* All-cells catch-up, row part (Proj.cpp:234-254): every row with
   pdt = simstep-1-ti > 0. */
__global__ void all_rows_kernel(const NetDev* __restrict__ net, const RunParams* __restrict__ rp, int p) {
  const ProjDev& J = net->projs[p];
  int simstep = rp->simstep0 - 1;
  float kp = J.taupdt * rp->old_prn;
  Coef k = make_coef(kp, J.ke, J.kzi, J.kzj, J.fp64);
  const float4* tab = rp->tabs[p].tab_old;
  int len = rp->tabs[p].old_len;
  int R = J.H * J.C;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    int pdt = simstep - J.ti[r];
    if (pdt > 0) {
      float pi = J.pi[r], ei = J.ei[r], zi = J.zi[r];
      float4 A, B;
      load_entry(tab, len, k, pdt, 2, A, B);
      row_decay(pi, ei, zi, k, A, B);
      J.pi[r] = pi;
      J.ei[r] = ei;
      J.zi[r] = zi;
      J.ti[r] = simstep;
    }
  }
}

/* All-cells catch-up, cell part (Proj.cpp:256-307).  Runs after
   all_rows_kernel so w_ij sees the updated pi. */
__global__ void all_cells_kernel(const NetDev* __restrict__ net, const RunParams* __restrict__ rp, int p) {
  const ProjDev& J = net->projs[p];
  int simstep = rp->simstep0 - 1;
  float kp = J.taupdt * rp->old_prn;
  Coef k = make_coef(kp, J.ke, J.kzi, J.kzj, J.fp64);
  const float4* tab = rp->tabs[p].tab_old;
  int len = rp->tabs[p].old_len;
  size_t ncell = (size_t)J.H * J.C * J.M;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (size_t)gridDim.x * blockDim.x) {
    int pdt = simstep - J.tij[c];
    if (pdt <= 0) {
      J.tij[c] = simstep;
    } else {
      float4 q = J.cell[c];
      float4 A, B;
      load_entry(tab, len, k, pdt, 0, A, B);
      cell_decay(q.x, q.y, q.z, q.w, k, A, B);
      J.cell[c] = q;
      J.tij[c] = simstep;
      if (kp != 0.0f) {
        int r = (int)(c / J.M);
        int j = (int)(c - (size_t)r * J.M);
        int h = r / J.C;
        float pi = J.pi[r];
        float pj = J.pj[h * J.M + j];
        J.wij[c] = J.wgain * dev_logf((q.x + J.eps2) / ((pi + J.eps) * (pj + J.eps)));
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* block helpers                                                              */
/* ------------------------------------------------------------------------ */

/* Ordered compaction over the kBlock threads: position of this thread's item
   among the set flags (in thread order) and, through *total, their number.
   Contains two __syncthreads; every thread of the block must call it. */
__device__ __forceinline__ int block_prefix(bool flag, int* s_warp, int* s_total, int* total) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned m = __ballot_sync(0xffffffffu, flag);
  int before = __popc(m & ((1u << lane) - 1u));
  if (lane == 0) s_warp[warp] = __popc(m);
  __syncthreads();
  if (warp == 0) {
    int c = lane < kWarps ? s_warp[lane] : 0;
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane < kWarps) s_warp[lane] = incl - c;
    if (lane == 31) *s_total = incl;
  }
  __syncthreads();
  int base = s_warp[warp];
  *total = *s_total;
  __syncwarp();
  return base + before;
}

/* maximum over the block (exact, order independent); one __syncthreads */
__device__ __forceinline__ float block_max(float v, float* s_red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    float w = __shfl_xor_sync(0xffffffffu, v, o);
    v = (w > v) ? w : v;
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) s_red[warp] = v;
  __syncthreads();
  float r = s_red[lane % kWarps];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    float w = __shfl_xor_sync(0xffffffffu, r, o);
    r = (w > r) ? w : r;
  }
  return r;
}

/* fill kernels used to (re)initialise the state on the device */
template <typename T>
__global__ void fill_kernel(T* p, size_t n, T v) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}

/* gather / scatter of one float of the (pij, eij, zi2, zj2) cells */
__global__ void cell_gather_kernel(const float4* cell, size_t n, int field, float* out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float4 v = cell[i];
    out[i] = field == 0 ? v.x : field == 1 ? v.y : field == 2 ? v.z : v.w;
  }
}

__global__ void cell_scatter_kernel(float4* cell, size_t n, int field, const float* in) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float4 v = cell[i];
    float x = in[i];
    if (field == 0) v.x = x; else if (field == 1) v.y = x; else if (field == 2) v.z = x; else v.w = x;
    cell[i] = v;
  }
}

/* Structural-plasticity pruning of one projection, one warp per row
   (ProcStructuralPlasticity/Prj.cpp:130-165 prune, :69-92 remove_conn).  A
   connected row (ii >= 0) goes when its row tick ti is below threshold_t, or
   when none of its weights reaches wp or wn (w >= wp or w <= wn; a NaN weight
   reaches neither).  A removed row gets ii = -1, di = 0, ti = 0, pi = 0,
   ei = 0 and pij = eij = zj2 = 0 in its cells; zi, zi2, tij, wij and the delay
   queue stay as they are, as in gsbn.  out[r] = the removed source MCU, or -1. */
__global__ void prune_rows_kernel(const ProjDev* __restrict__ projs, int p, int threshold_t, float wp, float wn,
                                  int* __restrict__ out) {
  const ProjDev& J = projs[p];
  const int R = J.H * J.C, M = J.M;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int r = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); r < R; r += nw) {
    const int src = J.ii[r];
    bool removed = false;
    if (src >= 0) {
      if (J.ti[r] < threshold_t) {
        removed = true;
      } else {
        bool strong = false;
        for (int j = lane; j < M; j += 32) {
          const float w = J.wij[(size_t)r * M + j];
          strong |= (w >= wp || w <= wn);
        }
        removed = !__any_sync(0xffffffffu, strong);
      }
    }
    if (removed) {
      for (int j = lane; j < M; j += 32) {
        float4 c = J.cell[(size_t)r * M + j];
        c.x = 0.0f; /* pij */
        c.y = 0.0f; /* eij */
        c.w = 0.0f; /* zj2 */
        J.cell[(size_t)r * M + j] = c;
      }
      if (lane == 0) {
        J.ii[r] = -1;
        J.di[r] = 0;
        J.ti[r] = 0;
        J.pi[r] = 0.0f;
        J.ei[r] = 0.0f;
      }
    }
    if (lane == 0) out[r] = removed ? src : -1;
  }
}

}  // namespace bcpnn

#endif /* BCPNN_DEVICE_CUH */
