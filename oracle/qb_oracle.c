/*
 * qb_oracle.c -- TEST INFRASTRUCTURE ONLY. The CPU oracle of the annealer.
 *
 * Only the tests, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load this library, and only as the checker. The product never calls it.
 *
 * Two groups of functions:
 *  1. Restatements of the reference's own algorithms (QuBLAR), each citing the
 *     file:line it follows. They are pinned bit-for-bit against the reference
 *     compiled from its sources (oracle/_ref) and against the reference's
 *     golden vectors (tests/golden).
 *  2. The coloured-Philox annealers: the same Metropolis rule and evaluators,
 *     visiting bits in the plan's colour-class order with Philox4x32-10 draws
 *     keyed by (seed, bit, sweep), and -- for the residual form -- the same
 *     fp32 operation order as the sm_100a kernels (lane-strided fmaf chains per
 *     bit joined by an xor butterfly). The GPU must match these bit-for-bit.
 *
 * Build: gcc -O2 -std=c11 -ffp-contract=off (no FMA contraction: every
 * expression rounds like the reference's host code).
 */
#include <math.h>
#include <stdint.h>

/* Lanes that share one bit's sum in the residual kernel (kGroup and kHeavy
 * in qublar_b200/csrc/qb_kernels.cu): a bit with more than ORC_HEAVY rays is
 * summed by 32 lanes, any other by ORC_GROUP -- the GPU's summation order. */
#define ORC_GROUP 8
#define ORC_HEAVY 64
/* Entries per segment of the lockstep kernel (kSeg in qb_kernels.cu). */
#define ORC_SEG 16
#include <stdlib.h>
#include <string.h>

/* ---- random numbers --------------------------------------------------------------- */

/* splitmix64 step and 53-bit uniform: ising_weighted.hpp:236-242
 * (identical to ising_recon.hpp:89-95). */
uint64_t orc_splitmix(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double orc_uniform(uint64_t* s) { return (double)(orc_splitmix(s) >> 11) * 0x1.0p-53; }

/* Philox4x32-10 from Salmon et al., SC'11 (section 4). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1, n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

uint64_t orc_draw_u53(uint64_t seed, uint32_t bit, uint32_t sweep, uint32_t stream) {
    const uint32_t ctr[4] = {bit, sweep, stream, 0u};
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    orc_philox4x32_10(ctr, key, o);
    return (((uint64_t)o[1] << 32) | (uint64_t)o[0]) >> 11;
}

/* The other half of the same block: the top 53 bits of words 3:2
 * (qb_philox.cuh draw_u53_pair). */
uint64_t orc_draw_u53_hi(uint64_t seed, uint32_t bit, uint32_t sweep, uint32_t stream) {
    const uint32_t ctr[4] = {bit, sweep, stream, 0u};
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    orc_philox4x32_10(ctr, key, o);
    return (((uint64_t)o[3] << 32) | (uint64_t)o[2]) >> 11;
}

/* Temperature of a sweep: ising_recon.hpp:129-131, ising_weighted.hpp:255-257. */
double orc_temperature(double t_hot, double t_cold, int anneal, int sweep) {
    const int den = anneal - 1 > 1 ? anneal - 1 : 1;
    double frac = (double)sweep / den;
    if (frac > 1.0) frac = 1.0;
    return sweep < anneal ? t_hot * pow(t_cold / t_hot, frac) : t_cold;
}

/* ---- integer Ising (ising_weighted.hpp) ------------------------------------------------ */

/* Symmetric CSR of an edge list in edge order: parse_rudy, ising_weighted.hpp:135-147. */
void orc_build_csr(int n, int64_t m, const int32_t* eu, const int32_t* ev, const int32_t* ew, int64_t* row,
                   int32_t* col, int32_t* w) {
    memset(row, 0, sizeof(int64_t) * (size_t)(n + 1));
    for (int64_t e = 0; e < m; ++e) { row[eu[e] + 1]++; row[ev[e] + 1]++; }
    for (int i = 0; i < n; ++i) row[i + 1] += row[i];
    int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    memcpy(fill, row, sizeof(int64_t) * (size_t)n);
    for (int64_t e = 0; e < m; ++e) {
        const int32_t a = eu[e], b = ev[e];
        col[fill[a]] = b; w[fill[a]++] = ew[e];
        col[fill[b]] = a; w[fill[b]++] = ew[e];
    }
    free(fill);
}

/* cut_of: ising_weighted.hpp:173-178. */
int64_t orc_cut_of(int64_t m, const int32_t* eu, const int32_t* ev, const int32_t* ew, const uint8_t* x) {
    int64_t cut = 0;
    for (int64_t e = 0; e < m; ++e)
        if (x[eu[e]] != x[ev[e]]) cut += ew[e];
    return cut;
}

/* energy_scratch: ising_weighted.hpp:181-189. */
int64_t orc_energy_scratch(int n, const int64_t* row, const int32_t* col, const int32_t* w, const uint8_t* x) {
    int64_t cut = 0;
    for (int i = 0; i < n; ++i)
        for (int64_t k = row[i]; k < row[i + 1]; ++k) {
            const int j = col[k];
            if (j > i && x[i] != x[j]) cut += w[k];
        }
    return -cut;
}

/* The maintained field f_i = sum_j w_ij s_j of a configuration (State::f,
 * ising_weighted.hpp:196), from scratch. */
void orc_fields(int n, const int64_t* row, const int32_t* col, const int32_t* w, const uint8_t* x, int64_t* f) {
    for (int i = 0; i < n; ++i) {
        int64_t acc = 0;
        for (int64_t k = row[i]; k < row[i + 1]; ++k) acc += (int64_t)w[k] * (x[col[k]] ? 1 : -1);
        f[i] = acc;
    }
}

typedef struct {
    int n;
    const int64_t* row;
    const int32_t* col;
    const int32_t* w;
    int8_t* s;
    int64_t* f;
    int64_t energy;
} orc_state;

/* State ctor, dE, flip: ising_weighted.hpp:199-217. */
static void st_init(orc_state* st) {
    for (int i = 0; i < st->n; ++i) {
        st->s[i] = -1;
        int64_t acc = 0;
        for (int64_t k = st->row[i]; k < st->row[i + 1]; ++k) acc -= st->w[k];
        st->f[i] = acc;
    }
    st->energy = 0;
}
static int64_t st_dE(const orc_state* st, int i) { return -(int64_t)st->s[i] * st->f[i]; }
static void st_flip(orc_state* st, int i) {
    const int64_t d = st_dE(st, i);
    const int64_t si = st->s[i];
    for (int64_t k = st->row[i]; k < st->row[i + 1]; ++k) st->f[st->col[k]] -= 2 * (int64_t)st->w[k] * si;
    st->s[i] = (int8_t)(-si);
    st->energy += d;
}

/* wising::anneal: ising_weighted.hpp:250-267 (sequential sweep, splitmix draw
 * only when dE > 0). trace (nullable) receives the tracked energy after each sweep. */
int64_t orc_wising_anneal(int n, const int64_t* row, const int32_t* col, const int32_t* w, double t_hot, double t_cold,
                          int anneal, int hold, uint64_t seed, uint8_t* x_out, double* trace) {
    orc_state st = {n, row, col, w, (int8_t*)malloc((size_t)n), (int64_t*)malloc(sizeof(int64_t) * (size_t)n), 0};
    st_init(&st);
    uint64_t state = seed * 0x2545F4914F6CDD1Dull + 1;
    const int total = anneal + hold;
    for (int sweep = 0; sweep < total; ++sweep) {
        const double temp = orc_temperature(t_hot, t_cold, anneal, sweep);
        for (int i = 0; i < n; ++i) {
            const double dE = (double)st_dE(&st, i);
            if (dE <= 0.0 || orc_uniform(&state) < exp(-dE / temp)) st_flip(&st, i);
        }
        if (trace) trace[sweep] = (double)st.energy;
    }
    for (int i = 0; i < n; ++i) x_out[i] = st.s[i] > 0 ? 1u : 0u;
    const int64_t e = st.energy;
    free(st.s);
    free(st.f);
    return e;
}

/* The coloured-Philox integer annealer: wising::anneal's Metropolis rule and
 * State, bits visited in colour-class order, draw = half `half` (0: words 1:0,
 * 1: words 3:2) of the Philox block of (seed, bit, sweep) -- replicas 2k and
 * 2k + 1 of a solve share a key and take one half each.
 * temps: the temperature of every sweep. */
int64_t orc_ising_anneal_coloured(int n, const int64_t* row, const int32_t* col, const int32_t* w,
                                  const int32_t* order, const double* temps, int sweeps, uint64_t seed, int half,
                                  uint8_t* x_out, int64_t* f_out, double* trace) {
    orc_state st = {n, row, col, w, (int8_t*)malloc((size_t)n), (int64_t*)malloc(sizeof(int64_t) * (size_t)n), 0};
    st_init(&st);
    for (int sweep = 0; sweep < sweeps; ++sweep) {
        const double T = temps[sweep];
        for (int k = 0; k < n; ++k) {
            const int i = order[k];
            const double dE = (double)st_dE(&st, i);
            if (dE <= 0.0) {
                st_flip(&st, i);
                continue;
            }
            const uint64_t u53 = half ? orc_draw_u53_hi(seed, (uint32_t)i, (uint32_t)sweep, 0u)
                                      : orc_draw_u53(seed, (uint32_t)i, (uint32_t)sweep, 0u);
            if ((double)u53 * 0x1.0p-53 < exp(-dE / T)) st_flip(&st, i);
        }
        if (trace) trace[sweep] = (double)st.energy;
    }
    for (int i = 0; i < n; ++i) {
        x_out[i] = st.s[i] > 0 ? 1u : 0u;
        if (f_out) f_out[i] = st.f[i];
    }
    const int64_t e = st.energy;
    free(st.s);
    free(st.f);
    return e;
}

/* Gray-code walk over all 2^n states (gset_bench.cu:288-309): tracked energy
 * and predicted dE against cut_of and energy_scratch at every state. Returns
 * the mismatch count; *best_cut receives the maximum cut. */
int64_t orc_gray_check(int n, int64_t m, const int32_t* eu, const int32_t* ev, const int32_t* ew, const int64_t* row,
                       const int32_t* col, const int32_t* w, int64_t* best_cut) {
    orc_state st = {n, row, col, w, (int8_t*)malloc((size_t)n), (int64_t*)malloc(sizeof(int64_t) * (size_t)n), 0};
    st_init(&st);
    uint8_t* x = (uint8_t*)calloc((size_t)n, 1);
    int64_t bad = 0, best = 0;
    const uint64_t states = (uint64_t)1 << n;
    for (uint64_t k = 1; k < states; ++k) {
        int bit = 0;
        while (!((k >> bit) & 1)) ++bit;
        const int64_t before = st.energy;
        const int64_t predicted = st_dE(&st, bit);
        st_flip(&st, bit);
        x[bit] ^= 1u;
        const int64_t cut = orc_cut_of(m, eu, ev, ew, x);
        if (st.energy != -cut || st.energy != orc_energy_scratch(n, row, col, w, x) || st.energy - before != predicted)
            ++bad;
        if (cut > best) best = cut;
    }
    if (best_cut) *best_cut = best;
    free(x);
    free(st.s);
    free(st.f);
    return bad;
}

/* ---- residual form (engine.hpp, ising_recon.hpp) -------------------------------------------- */

/* Field layout matches qb_residual_desc (include/qublar.h) and
 * argos::BinaryProblem (engine.hpp:30-49). */
typedef struct {
    int32_t n_vars;
    int32_t n_rays;
    const double* d;
    const double* w;
    const int32_t* row_ptr;
    const int32_t* ray;
    const float* a;
    const int32_t* nbr_ptr;
    const int32_t* nbr;
    double lambda;
    double kappa;
    const double* field;
} orc_resid;

static double lin_of(const orc_resid* p, int i) { return p->field ? p->field[i] : p->kappa; }   /* engine.hpp:47 */

/* binary_energy: ising_recon.hpp:65-79. */
double orc_binary_energy(const orc_resid* p, const uint8_t* x) {
    double* r = (double*)malloc(sizeof(double) * (size_t)(p->n_rays > 0 ? p->n_rays : 1));
    for (int b = 0; b < p->n_rays; ++b) r[b] = -p->d[b];
    double prior = 0.0;
    for (int i = 0; i < p->n_vars; ++i) {
        if (x[i])
            for (int k = p->row_ptr[i]; k < p->row_ptr[i + 1]; ++k) r[p->ray[k]] += p->a[k];
        prior += lin_of(p, i) * x[i];
        for (int k = p->nbr_ptr[i]; k < p->nbr_ptr[i + 1]; ++k)
            if (p->nbr[k] > i && x[p->nbr[k]] != x[i]) prior += p->lambda;
    }
    double data = 0.0;
    for (int b = 0; b < p->n_rays; ++b) data += 0.5 * p->w[b] * r[b] * r[b];
    free(r);
    return data + prior;
}

void orc_binary_energy_batch(const orc_resid* p, const uint8_t* X, int64_t K, double* e) {
    for (int64_t k = 0; k < K; ++k) e[k] = orc_binary_energy(p, X + (size_t)k * (size_t)p->n_vars);
}

/* local_field_dE: ising_recon.hpp:105-118. */
double orc_local_field_dE(const orc_resid* p, const uint8_t* x, const double* r, int i) {
    const double delta = x[i] ? -1.0 : 1.0;
    double dE = lin_of(p, i) * delta;
    for (int k = p->row_ptr[i]; k < p->row_ptr[i + 1]; ++k) {
        const double a = p->a[k] * delta;
        dE += p->w[p->ray[k]] * (r[p->ray[k]] * a + 0.5 * a * a);
    }
    for (int k = p->nbr_ptr[i]; k < p->nbr_ptr[i + 1]; ++k) {
        const int before = x[p->nbr[k]] != x[i];
        dE += p->lambda * (before ? -1.0 : 1.0);
    }
    return dE;
}

/* anneal_branch: ising_recon.hpp:121-144 (sequential sweep, splitmix draws,
 * double residuals). trace (nullable): binary_energy after each sweep, the
 * instrumentation of check_ree_qubo.cu:195-216. */
void orc_anneal_branch(const orc_resid* p, double t_hot, double t_cold, int anneal, int hold, uint64_t seed,
                       uint8_t* x, double* trace) {
    memset(x, 0, (size_t)p->n_vars);
    double* r = (double*)malloc(sizeof(double) * (size_t)(p->n_rays > 0 ? p->n_rays : 1));
    for (int b = 0; b < p->n_rays; ++b) r[b] = -p->d[b];
    uint64_t state = seed * 0x2545F4914F6CDD1Dull + 1;
    const int total = anneal + hold;
    for (int sweep = 0; sweep < total; ++sweep) {
        const double temp = orc_temperature(t_hot, t_cold, anneal, sweep);
        for (int i = 0; i < p->n_vars; ++i) {
            const double delta = x[i] ? -1.0 : 1.0;
            const double dE = orc_local_field_dE(p, x, r, i);
            if (dE <= 0.0 || orc_uniform(&state) < exp(-dE / temp)) {
                x[i] ^= 1u;
                for (int k = p->row_ptr[i]; k < p->row_ptr[i + 1]; ++k) r[p->ray[k]] += p->a[k] * delta;
            }
        }
        if (trace) trace[sweep] = orc_binary_energy(p, x);
    }
    free(r);
}

/* hi + lo += v with the fp32 rounding error carried in lo (TwoSum), the
 * compensated update of the GPU sweeps (qb_device.cuh two_sum_add). */
static void orc_two_sum(float* hi, float* lo, float v) {
    const float s = *hi + v;
    const float bp = s - *hi;
    const float e = (*hi - (s - bp)) + (v - bp);
    *hi = s;
    *lo = *lo + e;
}

/* The fp32 pair nearest an fp64 value: hi = fp32(v), lo = fp32(v - hi). */
static void orc_split(double v, float* hi, float* lo) {
    *hi = (float)v;
    *lo = (float)(v - (double)*hi);
}

/* The coloured-Philox residual annealer, in the fp32 operation order of the
 * sm_100a kernels. State per ray: the scaled residual rho_b = s_b (sum a x -
 * d_b), s_b = sqrt|w_b|, as an fp32 pair hi + lo; entry coefficient a' =
 * fp32(s_b a) (fp64 product rounded once) and sign(w_b); q_i = fp32(sum
 * sign(w) a'^2 / 2) summed in fp64 in entry order, lin_i = fp32(lin). h = sum
 * of sign(w) a' * fp32(hi + lo) over the bit's rays in the kernel's order:
 * mode 1 (lockstep) 16-entry segments added in order, each the fmaf chain over
 * its even entries plus the chain over its odd ones; mode 2 (cluster) G =
 * ORC_GROUP or 32 strided fmaf chains joined by an xor butterfly. dE =
 * ((delta * (lin + h)) + q) + lambda * (deg - 2 unlike); accept as
 * wising::anneal; a flip adds delta a' into each of its rays' pairs (TwoSum).
 * Every `refresh` sweeps rho is recomputed in fp64 (the ray's set bits in
 * ascending index, sum of fp64(a') minus s d) and split into the pair;
 * drift_out: max |fp64(hi) + fp64(lo) - rho|. trace (nullable): binary_energy
 * after each sweep; track (nullable): the energy of x = 0 plus the accepted dE
 * (fp64, visiting order) after each sweep. */
void orc_resid_anneal_coloured(const orc_resid* p, const int32_t* order, const double* temps, int sweeps, int refresh,
                               uint64_t seed, int mode, uint8_t* x, float* drift_out, double* trace, double* track) {
    const int n = p->n_vars, nr = p->n_rays;
    const int64_t nnz = p->row_ptr[n];
    float* hi = (float*)malloc(sizeof(float) * (size_t)(nr > 0 ? nr : 1));
    float* lo = (float*)malloc(sizeof(float) * (size_t)(nr > 0 ? nr : 1));
    double* sw = (double*)malloc(sizeof(double) * (size_t)(nr > 0 ? nr : 1));
    float* ap = (float*)malloc(sizeof(float) * (size_t)(nnz > 0 ? nnz : 1));   /* a' per bit-major entry */
    float* cf = (float*)malloc(sizeof(float) * (size_t)(nnz > 0 ? nnz : 1));   /* sign(w) a' */
    float* linf = (float*)malloc(sizeof(float) * (size_t)n);
    float* qf = (float*)malloc(sizeof(float) * (size_t)n);
    double e0 = 0.0;
    for (int b = 0; b < nr; ++b) {
        sw[b] = sqrt(fabs(p->w[b]));
        orc_split(-(sw[b] * p->d[b]), &hi[b], &lo[b]);
        e0 += 0.5 * p->w[b] * p->d[b] * p->d[b];
    }
    for (int i = 0; i < n; ++i) {
        double qd = 0.0;
        for (int k = p->row_ptr[i]; k < p->row_ptr[i + 1]; ++k) {
            const double w = p->w[p->ray[k]];
            ap[k] = (float)(sw[p->ray[k]] * (double)p->a[k]);
            cf[k] = w < 0.0 ? -ap[k] : ap[k];
            qd += (w < 0.0 ? -0.5 : 0.5) * (double)ap[k] * (double)ap[k];
        }
        qf[i] = (float)qd;
        linf[i] = (float)lin_of(p, i);
    }
    /* ray-major CSR, bits ascending */
    int32_t* rrow = (int32_t*)calloc((size_t)nr + 1, sizeof(int32_t));
    int32_t* rbit = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1));
    float* rap = (float*)malloc(sizeof(float) * (size_t)(nnz > 0 ? nnz : 1));
    for (int64_t k = 0; k < nnz; ++k) rrow[p->ray[k] + 1]++;
    for (int b = 0; b < nr; ++b) rrow[b + 1] += rrow[b];
    int32_t* fill = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nr > 0 ? nr : 1));
    memcpy(fill, rrow, sizeof(int32_t) * (size_t)nr);
    for (int i = 0; i < n; ++i)
        for (int k = p->row_ptr[i]; k < p->row_ptr[i + 1]; ++k) {
            const int32_t q = fill[p->ray[k]]++;
            rbit[q] = i;
            rap[q] = ap[k];
        }
    free(fill);
    memset(x, 0, (size_t)n);
    const float lam = (float)p->lambda;
    float drift = 0.0f;
    double E = e0;
    for (int sweep = 0; sweep < sweeps; ++sweep) {
        if (refresh > 0 && sweep > 0 && sweep % refresh == 0) {
            for (int b = 0; b < nr; ++b) {
                double acc = 0.0;
                for (int k = rrow[b]; k < rrow[b + 1]; ++k)
                    if (x[rbit[k]]) acc += (double)rap[k];
                const double v = acc - sw[b] * p->d[b];
                const float dv = (float)fabs(((double)hi[b] + (double)lo[b]) - v);
                if (dv > drift) drift = dv;
                orc_split(v, &hi[b], &lo[b]);
            }
        }
        const double T = temps[sweep];
        for (int kk = 0; kk < n; ++kk) {
            const int i = order[kk];
            float hl = 0.0f;
            if (mode == 1) {
                /* lockstep kernel: 16-entry segments in order; a segment's
                 * value is its even-entry fmaf chain plus its odd-entry chain */
                const int r0 = p->row_ptr[i], r1 = p->row_ptr[i + 1];
                for (int s0 = r0; s0 < r1; s0 += ORC_SEG) {
                    const int s1 = s0 + ORC_SEG < r1 ? s0 + ORC_SEG : r1;
                    float ev = 0.0f, od = 0.0f;
                    for (int k = s0; k < s1; k += 2) ev = fmaf(cf[k], hi[p->ray[k]] + lo[p->ray[k]], ev);
                    for (int k = s0 + 1; k < s1; k += 2) od = fmaf(cf[k], hi[p->ray[k]] + lo[p->ray[k]], od);
                    hl = hl + (ev + od);
                }
            }
            /* cluster kernel: G lanes, lane l sums entries l, l + G, ... as an
             * fmaf chain; an xor butterfly (G/2, ..., 1) joins them; lane 0 wins */
            const int G = mode == 1 ? 1 : (p->row_ptr[i + 1] - p->row_ptr[i] > ORC_HEAVY ? 32 : ORC_GROUP);
            float lane[32];
            for (int l = 0; l < G; ++l) lane[l] = 0.0f;
            for (int k = p->row_ptr[i]; k < p->row_ptr[i + 1]; ++k) {
                const int l = (k - p->row_ptr[i]) % G;
                lane[l] = fmaf(cf[k], hi[p->ray[k]] + lo[p->ray[k]], lane[l]);
            }
            for (int off = G / 2; off > 0; off >>= 1) {
                float nx[32];
                for (int l = 0; l < G; ++l) nx[l] = lane[l] + lane[l ^ off];
                memcpy(lane, nx, sizeof(float) * (size_t)G);
            }
            const float h = mode == 1 ? hl : lane[0];
            const uint8_t xi = x[i];
            int unlike = 0;
            for (int k = p->nbr_ptr[i]; k < p->nbr_ptr[i + 1]; ++k) unlike += x[p->nbr[k]] != xi;
            const int deg = p->nbr_ptr[i + 1] - p->nbr_ptr[i];
            const float delta = xi ? -1.0f : 1.0f;
            const float t = linf[i] + h;
            const float prior = lam * (float)(deg - 2 * unlike);
            const float dE = (delta * t + qf[i]) + prior;
            const double dEd = (double)dE;
            if (dEd <= 0.0 ||
                (double)orc_draw_u53(seed, (uint32_t)i, (uint32_t)sweep, 0u) * 0x1.0p-53 < exp(-dEd / T)) {
                for (int k = p->row_ptr[i]; k < p->row_ptr[i + 1]; ++k)
                    orc_two_sum(&hi[p->ray[k]], &lo[p->ray[k]], delta * ap[k]);
                x[i] = (uint8_t)(xi ^ 1u);
                E += dEd;
            }
        }
        if (trace) trace[sweep] = orc_binary_energy(p, x);
        if (track) track[sweep] = E;
    }
    if (drift_out) *drift_out = drift;
    free(hi); free(lo); free(sw); free(ap); free(cf); free(linf); free(qf); free(rrow); free(rbit); free(rap);
}

/* classify: ising_recon.hpp:305-309 (NotThere = 1, Exists = 0, Undecided = 2). */
void orc_classify(const float* p, int64_t n, float lo, float hi, uint8_t* out) {
    for (int64_t v = 0; v < n; ++v) out[v] = p[v] >= hi ? 1u : (p[v] <= lo ? 0u : 2u);
}

/* branch_fractions' reduction: ising_recon.hpp:160-163. */
void orc_fractions(const uint8_t* X, int R, int64_t n, float* frac) {
    for (int64_t i = 0; i < n; ++i) frac[i] = 0.0f;
    for (int b = 0; b < R; ++b)
        for (int64_t i = 0; i < n; ++i) frac[i] += X[(size_t)b * (size_t)n + (size_t)i];
    for (int64_t i = 0; i < n; ++i) frac[i] /= (float)R;
}

/* ---- weighted QUBO ------------------------------------------------------------------ */

/* E(x) = offset + sum_i h_i x_i + sum_e J_e x_u x_v in fp64: qubo_energy of
 * src/check_ree_qubo.cu:158-163 (offset + Qd over set bits + Qo over pairs of
 * set bits), summed sequentially. h may be NULL. */
double orc_qubo_energy(int n, int64_t m, const int32_t* eu, const int32_t* ev, const float* ew, const float* h,
                       double offset, const uint8_t* x) {
    double e = offset;
    if (h)
        for (int i = 0; i < n; ++i)
            if (x[i]) e += (double)h[i];
    for (int64_t k = 0; k < m; ++k)
        if (x[eu[k]] && x[ev[k]]) e += (double)ew[k];
    return e;
}


/* Mirror of the weighted-QUBO sweep of qublar_b200/csrc/qb_qubo.cu for one
 * replica: bits in colour-class order (order[k] = original bit at sweep
 * position k, classes class_ptr[0..nc]); a visit first adds the deltas of the
 * neighbours that flipped at their latest visit (CSR built from the edge list
 * in edge order, TwoSum into the fp32 pair hi + lo), every `refresh` sweeps
 * (sweep > 0) recomputes the field in fp64 and records |fp32 - fp64|, then
 * accepts if dE <= 0 or u53 * 2^-53 < exp(-dE / T), u53 the half `half` (0:
 * words 1:0, 1: words 3:2) of the Philox block of (seed, bit, sweep) -- the
 * kernel's replicas r and r + 32 share a key and take one half each. Returns
 * the tracked sum of accepted dE in fp64. */
double orc_qubo_anneal_coloured(int n, int64_t m, const int32_t* eu, const int32_t* ev, const float* ew,
                                const float* h, const int32_t* order, const int32_t* class_ptr, int nc,
                                const double* temps, int sweeps, int refresh, uint64_t seed, int half,
                                uint8_t* x_out, float* drift_out) {
    int64_t* row = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    for (int64_t e = 0; e < m; ++e) { row[eu[e] + 1]++; row[ev[e] + 1]++; }
    for (int i = 0; i < n; ++i) row[i + 1] += row[i];
    int32_t* col = (int32_t*)malloc(sizeof(int32_t) * (size_t)(2 * m + 1));
    float* w = (float*)malloc(sizeof(float) * (size_t)(2 * m + 1));
    int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
    for (int i = 0; i < n; ++i) fill[i] = row[i];
    for (int64_t e = 0; e < m; ++e) {
        col[fill[eu[e]]] = ev[e]; w[fill[eu[e]]++] = ew[e];
        col[fill[ev[e]]] = eu[e]; w[fill[ev[e]]++] = ew[e];
    }
    uint8_t* x = (uint8_t*)calloc((size_t)n, 1);
    uint8_t* f = (uint8_t*)calloc((size_t)n, 1);
    float* hi = (float*)malloc(sizeof(float) * (size_t)n);
    float* lo = (float*)calloc((size_t)n, sizeof(float));
    for (int i = 0; i < n; ++i) hi[i] = h ? h[i] : 0.0f;
    double track = 0.0;
    float drift = 0.0f;
    for (int sweep = 0; sweep < sweeps; ++sweep) {
        const double T = temps[sweep];
        const int fresh = refresh > 0 && sweep > 0 && sweep % refresh == 0;
        for (int c = 0; c < nc; ++c)
            for (int k = class_ptr[c]; k < class_ptr[c + 1]; ++k) {
                const int i = order[k];
                float H = hi[i], L = lo[i];
                double a = fresh ? (double)(h ? h[i] : 0.0f) : 0.0;
                for (int64_t e = row[i]; e < row[i + 1]; ++e) {
                    const int j = col[e];
                    if (f[j]) orc_two_sum(&H, &L, x[j] ? w[e] : -w[e]);
                    if (fresh && x[j]) a += (double)w[e];
                }
                if (fresh) {
                    const float d = (float)fabs((double)(H + L) - a);
                    if (d > drift) drift = d;
                    H = (float)a;
                    L = (float)(a - (double)H);
                }
                const float Lf = H + L;
                const float dE = x[i] ? -Lf : Lf;
                const uint64_t u53 = half ? orc_draw_u53_hi(seed, (uint32_t)i, (uint32_t)sweep, 0u)
                                          : orc_draw_u53(seed, (uint32_t)i, (uint32_t)sweep, 0u);
                const int acc = dE <= 0.0f || (double)u53 * 0x1.0p-53 < exp(-(double)dE / T);
                f[i] = (uint8_t)acc;
                if (acc) {
                    x[i] ^= 1u;
                    track += (double)dE;
                }
                hi[i] = H;
                lo[i] = L;
            }
    }
    memcpy(x_out, x, (size_t)n);
    if (drift_out) *drift_out = drift;
    free(row); free(col); free(w); free(fill); free(x); free(f); free(hi); free(lo);
    return track;
}
