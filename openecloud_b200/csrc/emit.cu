// emit.cu -- Furman-Pivi secondary emission and the uniform loader.
//
// Reference: particleEmitter.pyx FurmanEmitter.generateSecondaries (:154-308)
// and homoLoader (:41-72).  Two passes over the absorbed rows:
//  pass 1: primary energy and incidence angle, elastic/rediffused/true yields
//          and the number of secondaries drawn from P_n (:180-229);
//  scan:   output offsets of each absorbed particle's secondaries;
//  pass 2: energies (single secondary: elastic/rediffused/true split;
//          several: the joint energy split through I_x and P inverses,
//          :232-278) and cos-law directions about the wall normal (:280-302).
// Every absorbed particle draws from its own Philox stream, so the emitted
// set depends on the absorbed set, the run seed and the step only.
#include <math.h>
#include <stdint.h>

#include "oec_common.cuh"
#include "specfun.cuh"

namespace oec {
namespace {

constexpr int kDraws = 32;  // replay stride: uniforms per absorbed particle

struct Rec {
    double e0, dE, dR, pN1;
    int nsec;
};

// An absorbed row emits only with a finite position, energy and wall normal.
// A non-finite one (the reference would draw ten secondaries from NaN
// yields, each as non-finite, and so on at every step) emits nothing and is
// counted in status->n_emit_skipped.
__device__ __forceinline__ bool row_emits(const double *r, double e0, double n0, double n1) {
    return isfinite(r[0]) && isfinite(r[1]) && isfinite(e0) && isfinite(n0) && isfinite(n1);
}

__device__ __forceinline__ double clip(double x, double lo, double hi) {
    // particleEmitter.pyx:33-39 -- a NaN falls through to `hi`
    if (x <= hi && x >= lo) return x;
    if (x < lo) return lo;
    return hi;
}

__global__ void k_furman_pass1(oec_furman_t f, const double *__restrict__ rows, const double *__restrict__ normals,
                               const int32_t *n_abs, int cap, const int32_t *__restrict__ ids, uint2 key,
                               uint32_t step, const int32_t *step_dev, const double *__restrict__ replay,
                               Rec *__restrict__ rec,
                               int32_t *__restrict__ nsec, oec_status_t *status) {
    int na = min(*n_abs, cap);
    const double eFactor = 0.5 * f.particle_mass / 1.602176565e-19;
    int wd = 0, wt = 0;
    double lfac[11];  // lgamma(j + 1), j <= m <= 10, by the threads that have work
    if ((int)(blockIdx.x * blockDim.x + threadIdx.x) < na)
        for (int j = 0; j <= f.m; ++j) lfac[j] = sf::lgam((double)j + 1.0);
    int skipped = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < na; i += gridDim.x * blockDim.x) {
        const double *r = rows + 6 * (int64_t)i;
        const double n0 = normals[2 * i], n1 = normals[2 * i + 1];
        double v0 = sqrt(r[2] * r[2] + r[3] * r[3] + r[4] * r[4]);
        double e0 = eFactor * v0 * v0;
        if (!row_emits(r, e0, n0, n1)) {
            rec[i] = Rec{0., 0., 0., 1., 0};
            nsec[i] = 0;
            ++skipped;
            continue;
        }
        double th = acos((r[2] * n0 + r[3] * n1) / v0);
        if (th > 0.5 * sf::kPi) th = sf::kPi - th;
        th = clip(th, 0., f.theta0max);
        double ct = cos(th);
        double dE = (f.p1EInf + (f.p1Ehat - f.p1EInf) * exp(-pow(fabs(e0 - f.eEHat) / f.w, f.p) / f.p)) *
                    (1 + f.e1 * (1 - pow(ct, f.e2)));
        double dR = f.p1RInf * (1 - exp(-pow(e0 / f.eR, f.r))) * (1 + f.r1 * (1 - pow(ct, f.r2)));
        double eHat = f.eHat0 * (1 + f.t3 * (1 - pow(ct, f.t4)));
        double dTS0 = f.deltaTSHat * f.s * e0 / eHat / (f.s - 1 + pow(e0 / eHat, f.s));
        double dTS = dTS0 * (1 + f.t1 * (1 - pow(ct, f.t2)));
        double sum = dE + dR;
        if (sum >= f.deltaERmax) {
            dE = dE / sum * f.deltaERmax;
            dR = dR / sum * f.deltaERmax;
            ++wd;
        }
        double dTSp = dTS / (1 - dE - dR);
        if (dTSp >= f.m) {
            dTSp = f.m;
            ++wt;
        } else if (dTSp < 0) {
            dTSp = 0;
        }
        double pr = dTSp / f.m;
        double keep = 1 - dE - dR;
        sf::Draws dr{key, ids ? (uint32_t)ids[i] : (uint32_t)i, step + (step_dev ? (uint32_t)*step_dev : 0u),
                     replay ? replay + (int64_t)i * kDraws : nullptr};
        double u = dr.next();
        // P_n = binom(n; m, pr) (1 - dE - dR), P_1 += dE + dR (:217-221);
        // inverse-CDF draw over n < m, default m (:222-229)
        // binom_pdf(k; m, pr) with lgamma(j+1) and the logs of pr evaluated once
        // (the same values as sf::binom_pdf)
        const double lp = log(pr), l1p = log1p(-pr);
        auto pdf = [&](unsigned k) -> double {
            const unsigned m = (unsigned)f.m;
            if (pr == 0.0) return k == 0 ? 1.0 : 0.0;
            if (pr == 1.0) return k == m ? 1.0 : 0.0;
            const double lc = lfac[m] - lfac[k] - lfac[m - k];
            return exp(lc + k * lp + (double)(m - k) * l1p);
        };
        const double pN1 = pdf(1u) * keep + (dE + dR);
        int n = f.m;
        double cum = 0.0;
        for (int k = 0; k < f.m; ++k) {
            cum += (k == 1) ? pN1 : pdf((unsigned)k) * keep;
            if (u <= cum) {
                n = k;
                break;
            }
        }
        rec[i] = Rec{e0, dE, dR, pN1, n};
        nsec[i] = n;
    }
    if (wd) atomicAdd(&status->warn_derm, wd);
    if (wt) atomicAdd(&status->warn_tsprime, wt);
    if (skipped) atomicAdd(&status->n_emit_skipped, skipped);
}

// Pass 2a: the costly inverses of the joint energy split of a multi-secondary
// emission (particleEmitter.pyx:255-266), one thread per (absorbed particle,
// slot).  For n secondaries slot k < n-1 holds theta_k =
// asin(sqrt(I^-1_u(P(n-k-1), P))) from draw 1+k and slot n-1 holds
// y = sqrt(P^-1(nP, u p0)) from draw n: the same draws and the same
// arithmetic as one thread doing them in sequence, but the n calls run side
// by side instead of one after the other.
constexpr int kSlots = 10;

__global__ void k_furman_pass2a(oec_furman_t f, const int32_t *n_abs, int cap, const int32_t *__restrict__ ids,
                                uint2 key, uint32_t step, const int32_t *step_dev, const double *__restrict__ replay,
                                const Rec *__restrict__ rec, double *__restrict__ split) {
    const int na = min(*n_abs, cap);
    const int total = na * kSlots;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int i = t / kSlots, k = t % kSlots;
        const Rec R = rec[i];
        const int n = R.nsec;
        if (n < 2 || k >= n) continue;
        const double P = f.pSmallN[n - 1], eps = f.epsN[n - 1];
        sf::Draws dr{key, ids ? (uint32_t)ids[i] : (uint32_t)i, step + (step_dev ? (uint32_t)*step_dev : 0u),
                     replay ? replay + (int64_t)i * kDraws : nullptr};
        dr.d = 1 + k;
        double v;
        if (k < n - 1) {
            v = asin(sqrt(sf::betaincinv(P * (n - k - 1), P, dr.next())));
        } else {
            const double p0 = sf::gammainc(n * P, R.e0 / eps);
            v = sqrt(sf::gammaincinv(n * P, dr.next() * p0));
        }
        split[(int64_t)i * kSlots + k] = v;
    }
}

__global__ void k_furman_pass2(oec_furman_t f, const double *__restrict__ rows, const double *__restrict__ normals,
                               const int32_t *n_abs, int cap, const int32_t *__restrict__ ids, uint2 key,
                               uint32_t step, const int32_t *step_dev, const double *__restrict__ replay,
                               const Rec *__restrict__ rec, const double *__restrict__ split,
                               const int32_t *__restrict__ offset, double *__restrict__ out, int out_cap,
                               oec_status_t *status) {
    int na = min(*n_abs, cap);
    if (na <= 0) return;
    const double eFactorInv = 1.0 / (0.5 * f.particle_mass / 1.602176565e-19);
    const Rec last = rec[na - 1];
    int dropped = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < na; i += gridDim.x * blockDim.x) {
        const Rec R = rec[i];
        const int n = R.nsec;
        if (n == 0) continue;
        const double *r = rows + 6 * (int64_t)i;
        const double n0 = normals[2 * i], n1 = normals[2 * i + 1];
        sf::Draws dr{key, ids ? (uint32_t)ids[i] : (uint32_t)i, step + (step_dev ? (uint32_t)*step_dev : 0u),
                     replay ? replay + (int64_t)i * kDraws : nullptr};
        dr.d = 1;  // draw 0 was the secondary count
        double eSec[10];
        const double e0 = R.e0;
        if (n == 1) {
            // compat: the reference reads the split of the LAST absorbed particle
            // of pass 1 (stale loop variables, particleEmitter.pyx:245-246)
            const Rec &S = f.compat_last ? last : R;
            double aE = S.dE / S.pN1, aR = S.dR / S.pN1;
            double u = dr.next();
            if (u < aE) {
                double sig = f.scaleSigmaE ? f.sigmaE * sqrt(e0 / 300) : f.sigmaE;
                eSec[0] = e0 - fabs(sig * dr.normal());
                if (eSec[0] < 0.) eSec[0] = dr.next() * e0;
            } else if (u < aE + aR) {
                eSec[0] = e0 * pow(dr.next(), 1. / (1. + f.q));
            } else {
                eSec[0] = f.epsN[0] * sf::gammaincinv(f.pSmallN[0], dr.next() * sf::gammainc(f.pSmallN[0], e0 / f.epsN[0]));
            }
        } else {
            // theta_k and y from pass 2a (draws 1 .. n)
            const double *sp = split + (int64_t)i * kSlots;
            const double eps = f.epsN[n - 1];
            double th[10];
            for (int k = 0; k < n - 1; ++k) th[k] = sp[k];
            const double y = sp[n - 1];
            dr.d = n + 1;
            double yk[10];
            yk[0] = y * cos(th[0]);
            yk[n - 1] = y;
            for (int k = 0; k < n - 1; ++k) yk[n - 1] *= sin(th[k]);
            for (int k = 1; k < n - 1; ++k) {
                yk[k] = y * cos(th[k]);
                for (int t = 0; t < k; ++t) yk[k] *= sin(th[t]);
            }
            for (int k = 0; k < n; ++k) eSec[k] = eps * (yk[k] * yk[k]);
        }
        int o = offset[i];
        for (int k = 0; k < n; ++k) {
            double vs = sqrt(eFactorInv * eSec[k]);
            double thS = asin(dr.next());
            double cT = cos(thS), sT = sin(thS);
            double phS = dr.next() * sf::kPi * 2.;
            double cP = cos(phS), sP = sin(phS);
            double t1 = cT * n0 - sT * n1;
            double t2 = sT * n0 + cT * n1;
            if (o + k >= out_cap) {
                ++dropped;
                continue;
            }
            double *q = out + 6 * (int64_t)(o + k);
            q[0] = r[0];
            q[1] = r[1];
            q[2] = vs * ((cP + n0 * n0 * (1 - cP)) * t1 + n0 * n1 * (1 - cP) * t2);
            q[3] = vs * ((cP + n1 * n1 * (1 - cP)) * t2 + n0 * n1 * (1 - cP) * t1);
            q[4] = vs * (-sP * n1 * t1 + sP * n0 * t2);
            q[5] = r[5];
        }
    }
    if (dropped) atomicAdd(&status->n_capacity_drop, dropped);
}

// ------------------------------------------------------------------ scan

constexpr int kScanT = 1024;
constexpr int kMaxAbsorbedRows = 1 << 26;

// Blocks of the two-level count scan (at least kScanT partial slots).
inline int scan_blocks(int cap) {
    const int nb = (cap + kScanT - 1) / kScanT;
    return nb > kScanT ? nb : kScanT;
}

__device__ __forceinline__ int block_scan_excl(int v, int *tot, int *sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(kFullMask, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int s = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(kFullMask, s, o);
            if (lane >= o) s += y;
        }
        sh[lane] = s;
    }
    __syncthreads();
    int before = (wid > 0 ? sh[wid - 1] : 0) + x - v;
    if (tot) *tot = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before;
}

__global__ void k_scan_blocks(const int32_t *in, const int32_t *n_p, int cap, int32_t *out, int *partial) {
    __shared__ int sh[32];
    int n = min(*n_p, cap);
    int i = blockIdx.x * kScanT + threadIdx.x;
    int v = i < n ? in[i] : 0;
    int tot;
    int ex = block_scan_excl(v, &tot, sh);
    if (i < cap) out[i] = ex;
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

// Exclusive scan of the nb block totals by one CTA, kScanT at a time with a
// running carry.
__global__ void k_scan_partials(int *partial, int nb, int32_t *total) {
    __shared__ int sh[32];
    int carry = 0;
    for (int base = 0; base < nb; base += kScanT) {
        const int i = base + threadIdx.x;
        const int v = i < nb ? partial[i] : 0;
        int tot;
        const int ex = block_scan_excl(v, &tot, sh);
        if (i < nb) partial[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan_add(int32_t *out, const int32_t *n_p, int cap, const int *partial) {
    int n = min(*n_p, cap);
    int i = blockIdx.x * kScanT + threadIdx.x;
    if (i < n) out[i] += partial[blockIdx.x];
}

// The same scan in one CTA when the row capacity is small (a buildup step
// absorbs a few hundred rows of a capacity of tens of thousands): the first
// n rows, kScanT at a time with a running carry, one launch instead of three.
// Rows past n keep what they held; the emission passes read only rows < n.
constexpr int kSmallScanBlocks = 32;

__global__ void __launch_bounds__(kScanT)
    k_scan_small(const int32_t *in, const int32_t *n_p, int cap, int32_t *out, int32_t *total) {
    __shared__ int sh[32];
    const int n = min(*n_p, cap);
    int carry = 0;
    for (int base = 0; base < n; base += kScanT) {  // same trip count in every thread
        const int i = base + threadIdx.x;
        const int v = i < n ? in[i] : 0;
        int tot;
        const int ex = block_scan_excl(v, &tot, sh);
        if (i < n) out[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) *total = carry;
}

// offsets of the rows' secondaries and their total
void scan_counts(const int32_t *nsec, const int32_t *n_abs_dev, int cap, int32_t *off, int *partial,
                 int32_t *n_out_dev, cudaStream_t s) {
    const int nblocks = (cap + kScanT - 1) / kScanT;
    if (nblocks <= kSmallScanBlocks) {
        k_scan_small<<<1, kScanT, 0, s>>>(nsec, n_abs_dev, cap, off, n_out_dev);
        return;
    }
    k_scan_blocks<<<nblocks, kScanT, 0, s>>>(nsec, n_abs_dev, cap, off, partial);
    k_scan_partials<<<1, kScanT, 0, s>>>(partial, nblocks, n_out_dev);
    k_scan_add<<<nblocks, kScanT, 0, s>>>(off, n_abs_dev, cap, partial);
}

// ------------------------------------------- simplified emitters
// SecElecEmitter (particleEmitter.pyx:355-484) and SimpleSecEmitter
// (:506-597): pass 1 draws the elastic / rediffused / true counts (draws
// 0, 1, 2), the scan places each row's secondaries, pass 2 writes them
// (draws from 3 on, in the reference's order).
constexpr int kSecDraws = 64;  // replay stride: uniforms per absorbed row

struct SRec {
    double e0;
    int nE, nR, nT, pad;
};

__global__ void k_secelec_pass1(oec_secelec_t f, const double *__restrict__ rows, const double *__restrict__ normals,
                                const int32_t *n_abs, int cap, const int32_t *__restrict__ ids, uint2 key,
                                uint32_t step, const int32_t *step_dev, const double *__restrict__ replay,
                                SRec *__restrict__ rec, int32_t *__restrict__ nsec, oec_status_t *status) {
    const int na = min(*n_abs, cap);
    const double mass = f.model == 1 ? 9.10938291e-31 : f.particle_mass;
    const double eF = 0.5 * mass / 1.602176565e-19;
    int capped = 0, skipped = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < na; i += gridDim.x * blockDim.x) {
        const double *r = rows + 6 * (int64_t)i;
        const double v0 = sqrt(r[2] * r[2] + r[3] * r[3] + r[4] * r[4]);
        const double e0 = eF * v0 * v0;
        if (!row_emits(r, e0, normals[2 * i], normals[2 * i + 1])) {
            rec[i] = SRec{0., 0, 0, 0, 0};
            nsec[i] = 0;
            ++skipped;
            continue;
        }
        double dE, dR, dTS;
        if (f.model == 1) {
            const double s = 1.813, eHat = 310;
            dE = 0.05;
            dR = 0.5;
            dTS = 1.4 * s * e0 / eHat / (s - 1 + pow(e0 / eHat, s));
        } else {
            double th = acos((r[2] * normals[2 * i] + r[3] * normals[2 * i + 1]) / v0);
            if (th > 0.5 * sf::kPi) th = sf::kPi - th;
            th = clip(th, 0., f.theta0max);
            const double ct = cos(th);
            dE = (f.p1EInf + (f.p1Ehat - f.p1EInf) * exp(-pow(fabs(e0 - f.eEHat) / f.w, f.p) / f.p)) *
                 (1 + f.e1 * (1 - pow(ct, f.e2)));
            dR = f.p1RInf * (1 - exp(-pow(e0 / f.eR, f.r))) * (1 + f.r1 * (1 - pow(ct, f.r2)));
            const double eHat = f.eHat0 * (1 + f.t3 * (1 - pow(ct, f.t4)));
            dTS = f.deltaTSHat * f.s * e0 / eHat / (f.s - 1 + pow(e0 / eHat, f.s)) * (1 + f.t1 * (1 - pow(ct, f.t2)));
            const double t = dE + dR;
            if (t >= f.deltaERmax) {
                dE = dE / t * f.deltaERmax;
                dR = dR / t * f.deltaERmax;
            }
        }
        sf::Draws dr{key, ids ? (uint32_t)ids[i] : (uint32_t)i, step + (step_dev ? (uint32_t)*step_dev : 0u),
                     replay ? replay + (int64_t)i * kSecDraws : nullptr};
        const int nE = dr.next() <= dE ? 1 : 0;
        const int nR = dr.next() <= dR ? 1 : 0;
        // <unsigned int> truncation of the reference (:391, :553), then +1
        // with the probability of the fraction; a huge yield is capped below
        int nT = dTS >= 1e9 ? 1000000000 : (dTS > 0.0 ? (int)dTS : 0);
        if (dr.next() <= dTS - nT) ++nT;
        if (nT > f.max_ts) {
            nT = f.max_ts;
            ++capped;
        }
        rec[i] = SRec{e0, nE, nR, nT, 0};
        nsec[i] = nE + nR + nT;
    }
    if (capped) atomicAdd(&status->warn_tsprime, capped);
    if (skipped) atomicAdd(&status->n_emit_skipped, skipped);
}

__device__ __forceinline__ void put_row(double *q, const double *r, double vx, double vy, double vz) {
    q[0] = r[0];
    q[1] = r[1];
    q[2] = vx;
    q[3] = vy;
    q[4] = vz;
    q[5] = r[5];
}

__global__ void k_secelec_pass2(oec_secelec_t f, const double *__restrict__ rows, const double *__restrict__ normals,
                                const int32_t *n_abs, int cap, const int32_t *__restrict__ ids, uint2 key,
                                uint32_t step, const int32_t *step_dev, const double *__restrict__ replay,
                                const SRec *__restrict__ rec, const int32_t *__restrict__ offset,
                                double *__restrict__ out, int out_cap, oec_status_t *status) {
    const int na = min(*n_abs, cap);
    const double mass = f.model == 1 ? 9.10938291e-31 : f.particle_mass;
    const double eFi = 1.0 / (0.5 * mass / 1.602176565e-19);
    int dropped = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < na; i += gridDim.x * blockDim.x) {
        const SRec R = rec[i];
        if (R.nE + R.nR + R.nT == 0) continue;
        const double *r = rows + 6 * (int64_t)i;
        sf::Draws dr{key, ids ? (uint32_t)ids[i] : (uint32_t)i, step + (step_dev ? (uint32_t)*step_dev : 0u),
                     replay ? replay + (int64_t)i * kSecDraws : nullptr};
        dr.d = 3;  // draws 0..2 were the counts
        int o = offset[i];
        auto slot = [&](void) -> double * {
            if (o >= out_cap) {
                ++dropped;
                ++o;
                return nullptr;
            }
            return out + 6 * (int64_t)(o++);
        };
        if (R.nE) {
            if (double *q = slot()) put_row(q, r, -r[2], -r[3], -r[4]);
        }
        if (R.nR) {
            const double u = dr.next();
            const double vF = f.model == 1 ? sqrt(u) : sqrt(pow(u, 1. / (1. + f.q)));
            if (double *q = slot()) put_row(q, r, -r[2] * vF, -r[3] * vF, -r[4] * vF);
        }
        const int n = R.nT;
        if (n <= 0) continue;
        double eSec[10];
        if (f.model == 1) {
            for (int k = 0; k < n; ++k) eSec[k] = dr.next() * 5;
            for (int k = 0; k < n; ++k) {
                const double vF = sqrt(eSec[k] / R.e0);
                if (double *q = slot()) put_row(q, r, -r[2] * vF, -r[3] * vF, -r[4] * vF);
            }
            continue;
        }
        double eSum = 0.;
        for (int k = 0; k < n; ++k) {
            eSec[k] = exp(f.sigmaETS * dr.normal() + f.muETS);
            eSum += eSec[k];
        }
        if (eSum > R.e0)
            for (int k = 0; k < n; ++k) eSec[k] = dr.next() * R.e0 / n;
        const double n0 = normals[2 * i], n1 = normals[2 * i + 1];
        for (int k = 0; k < n; ++k) {
            const double vs = sqrt(eFi * eSec[k]);
            const double thS = asin(dr.next());
            const double cT = cos(thS), sT = sin(thS);
            const double phS = dr.next() * sf::kPi * 2.;
            const double cP = cos(phS), sP = sin(phS);
            const double t1 = cT * n0 - sT * n1, t2 = sT * n0 + cT * n1;
            if (double *q = slot())
                put_row(q, r, vs * ((cP + n0 * n0 * (1 - cP)) * t1 + n0 * n1 * (1 - cP) * t2),
                        vs * ((cP + n1 * n1 * (1 - cP)) * t2 + n0 * n1 * (1 - cP) * t1),
                        vs * (-sP * n1 * t1 + sP * n0 * t2));
        }
    }
    if (dropped) atomicAdd(&status->n_capacity_drop, dropped);
}

// ---------------------------------------------------------- homoLoader

// Rejection sampling of uniform positions inside the boundary
// (particleEmitter.pyx:52-63) with Philox draws: particle i tries
// candidate points until one is inside (at most `max_tries`).
__global__ void k_homo_load(oec_particles_t p, int64_t n, int kind, double lx, double ly, const uint16_t *faces,
                           const double *bpts, const int32_t *cpi, double lxh_ext, double lyh_ext, double dx,
                           double dy, int nx, int ny, double w0, double vsigma, int randomize_weight, uint2 key,
                           int max_tries, int32_t *failed) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        sf::Draws dr{key, (uint32_t)i, 0xffffffffu, nullptr};
        double x = 0, y = 0;
        bool ok = false;
        for (int t = 0; t < max_tries && !ok; ++t) {
            x = (dr.next() - 0.5) * lx;
            y = (dr.next() - 0.5) * ly;
            if (kind == OEC_BOUNDARY_RECT) {
                ok = !(x < -lx * 0.5 || x > lx * 0.5 || y < -ly * 0.5 || y > ly * 0.5);
            } else if (kind == OEC_BOUNDARY_ELLIPSE) {
                ok = !(x * x * (4. / (lx * lx)) + y * y * (4. / (ly * ly)) >= 1.);
            } else {
                int ix = (int)((x + lxh_ext) * (1. / dx)), iy = (int)((y + lyh_ext) * (1. / dy));
                int c = ix + iy * nx;
                unsigned fc = faces[c];
                if (fc == 8) ok = true;
                else if (fc == 0) ok = false;
                else {
                    int a = cpi[2 * c], b = cpi[2 * c + 1];
                    ok = a >= 0 && b >= 0 &&
                         (bpts[2 * a] - x) * (bpts[2 * b + 1] - y) > (bpts[2 * b] - x) * (bpts[2 * a + 1] - y);
                }
            }
        }
        if (!ok) atomicAdd(failed, 1);
        double ux = (x + lxh_ext) * (1. / dx), uy = (y + lyh_ext) * (1. / dy);
        int ix = (int)fmax(fmin(floor(ux), (double)(nx - 2)), 0.0);
        int iy = (int)fmax(fmin(floor(uy), (double)(ny - 2)), 0.0);
        p.cell[i] = ix + iy * nx;
        p.ox[i] = fminf(fmaxf((float)(ux - ix), 0.f), 0x1.fffffep-1f);
        p.oy[i] = fminf(fmaxf((float)(uy - iy), 0.f), 0x1.fffffep-1f);
        p.vx[i] = (float)(dr.normal() * vsigma);
        p.vy[i] = (float)(dr.normal() * vsigma);
        p.vz[i] = (float)(dr.normal() * vsigma);
        p.w[i] = (float)(randomize_weight ? w0 * (0.5 + dr.next()) : w0);
    }
}

}  // namespace
}  // namespace oec

using namespace oec;

extern "C" int oec_furman_emit(const oec_furman_t *params, const double *rows_dev, const double *normals_dev,
                               const int32_t *n_abs_dev, int32_t cap, const int32_t *ids_dev, uint64_t seed,
                               uint32_t step, const int32_t *step_dev, const double *replay_uniforms_dev,
                               void *work_dev,
                               double *out_rows_dev, int32_t out_cap, int32_t *n_out_dev, oec_status_t *status_dev,
                               void *stream) {
    if (!params || !rows_dev || !normals_dev || !n_abs_dev || !work_dev || !out_rows_dev || !n_out_dev ||
        !status_dev || cap < 0 || out_cap < 0 || params->m < 1 || params->m > 10)
        return OEC_ERR_INVALID;
    if (cap > kMaxAbsorbedRows) return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    // work layout: Rec[cap] | split[cap * kSlots] (f64) | nsec[cap] | offset[cap] | partial[scan_blocks(cap)]
    char *w = static_cast<char *>(work_dev);
    Rec *rec = reinterpret_cast<Rec *>(w);
    double *split = reinterpret_cast<double *>(w + sizeof(Rec) * (size_t)cap);
    int32_t *nsec = reinterpret_cast<int32_t *>(split + (size_t)cap * kSlots);
    int32_t *off = nsec + cap;
    int *partial = off + cap;
    uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    int g = persistent_grid((cap + 127) / 128, 8);
    k_furman_pass1<<<g, 128, 0, s>>>(*params, rows_dev, normals_dev, n_abs_dev, cap, ids_dev, key, step, step_dev,
                                     replay_uniforms_dev, rec, nsec, status_dev);
    if (cap > 0) {
        scan_counts(nsec, n_abs_dev, cap, off, partial, n_out_dev, s);
    } else {
        OEC_CUDA_TRY(cudaMemsetAsync(n_out_dev, 0, sizeof(int32_t), s));
    }
    k_furman_pass2a<<<persistent_grid(((int64_t)cap * kSlots + 127) / 128, 8), 128, 0, s>>>(
        *params, n_abs_dev, cap, ids_dev, key, step, step_dev, replay_uniforms_dev, rec, split);
    k_furman_pass2<<<g, 128, 0, s>>>(*params, rows_dev, normals_dev, n_abs_dev, cap, ids_dev, key, step, step_dev,
                                     replay_uniforms_dev, rec, split, off, out_rows_dev, out_cap, status_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int oec_secelec_emit(const oec_secelec_t *params, const double *rows_dev, const double *normals_dev,
                                const int32_t *n_abs_dev, int32_t cap, const int32_t *ids_dev, uint64_t seed,
                                uint32_t step, const int32_t *step_dev, const double *replay_uniforms_dev,
                                void *work_dev, double *out_rows_dev, int32_t out_cap, int32_t *n_out_dev,
                                oec_status_t *status_dev, void *stream) {
    if (!params || !rows_dev || !normals_dev || !n_abs_dev || !work_dev || !out_rows_dev || !n_out_dev ||
        !status_dev || cap < 0 || out_cap < 0 || params->model < 0 || params->model > 1 || params->max_ts < 1 ||
        params->max_ts > 10 || cap > kMaxAbsorbedRows)
        return OEC_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    // work layout: SRec[cap] | nsec[cap] | offset[cap] | partial[scan_blocks(cap)]
    char *w = static_cast<char *>(work_dev);
    SRec *rec = reinterpret_cast<SRec *>(w);
    int32_t *nsec = reinterpret_cast<int32_t *>(w + sizeof(SRec) * (size_t)cap);
    int32_t *off = nsec + cap;
    int *partial = off + cap;
    const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    const int g = persistent_grid((cap + 127) / 128, 8);
    k_secelec_pass1<<<g, 128, 0, s>>>(*params, rows_dev, normals_dev, n_abs_dev, cap, ids_dev, key, step, step_dev,
                                      replay_uniforms_dev, rec, nsec, status_dev);
    if (cap > 0) {
        scan_counts(nsec, n_abs_dev, cap, off, partial, n_out_dev, s);
    } else {
        OEC_CUDA_TRY(cudaMemsetAsync(n_out_dev, 0, sizeof(int32_t), s));
    }
    k_secelec_pass2<<<g, 128, 0, s>>>(*params, rows_dev, normals_dev, n_abs_dev, cap, ids_dev, key, step, step_dev,
                                      replay_uniforms_dev, rec, off, out_rows_dev, out_cap, status_dev);
    OEC_LAUNCH_CHECK();
    return OEC_OK;
}

extern "C" int64_t oec_secelec_work_bytes(int32_t cap) {
    if (cap < 0 || cap > kMaxAbsorbedRows) return -1;
    return (int64_t)sizeof(SRec) * cap + 2 * sizeof(int32_t) * (int64_t)cap + sizeof(int) * (int64_t)scan_blocks(cap) +
           256;
}

extern "C" int64_t oec_furman_work_bytes(int32_t cap) {
    if (cap < 0 || cap > kMaxAbsorbedRows) return -1;
    return (int64_t)sizeof(Rec) * cap + (int64_t)sizeof(double) * kSlots * cap + 2 * sizeof(int32_t) * (int64_t)cap +
           sizeof(int) * (int64_t)scan_blocks(cap) + 256;
}

extern "C" int oec_homo_load(const oec_grid_t *grid, const oec_boundary_t *boundary, oec_particles_t *p, int64_t n,
                             double weight, double vsigma, int32_t randomize_weight, uint64_t seed,
                             int32_t *failed_dev, void *stream) {
    if (!grid || !boundary || !p || n < 0 || n > p->capacity || !failed_dev) return OEC_ERR_INVALID;
    GridConst gc = make_grid_const(*grid);
    cudaStream_t s = as_stream(stream);
    int32_t cnt = (int32_t)n;
    OEC_CUDA_TRY(cudaMemsetAsync(failed_dev, 0, sizeof(int32_t), s));
    uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    k_homo_load<<<persistent_grid((n + 255) / 256, 8), 256, 0, s>>>(
        *p, n, boundary->kind, gc.lx, gc.ly, boundary->inside_faces_dev, boundary->boundary_points_dev,
        boundary->cut_cell_points_ind_dev, gc.lxh, gc.lyh, gc.dx, gc.dy, gc.nx, gc.ny, weight, vsigma,
        randomize_weight, key, 1000, failed_dev);
    OEC_LAUNCH_CHECK();
    OEC_CUDA_TRY(cudaMemcpyAsync(p->count, &cnt, sizeof(int32_t), cudaMemcpyHostToDevice, s));
    OEC_CUDA_TRY(cudaStreamSynchronize(s));  // `cnt` lives on this stack frame
    return OEC_OK;
}
