// Provable-rock freezing of a residual-form problem on the device: the
// pre-pass of freeze_provable_rock (src/ising_recon.hpp:168-235).
//
// For a 0 -> 1 flip of bit i, whatever the other bits do,
//   dE >= sum_b w_b a_bi (a_bi / 2 - d_b) + lin_i + lambda (#frozen - #free neighbours);
// a bit whose bound reaches `margin` is rock in every branch that matters and
// is fixed at 0. Freezing tightens the neighbours' bounds, so the test repeats
// to a fixpoint. With lambda >= 0 every bound only grows as bits freeze, so
// the fixpoint (the least set closed under the test) does not depend on the
// visiting order: the device runs Jacobi rounds over all bits at once and
// reaches the set the reference's sequential rounds reach. The bounds are
// evaluated in fp64 in the reference's operation order without fused
// multiply-adds, so every comparison is the reference's. The reduced problem
// (the bits that can still change, bonds to frozen rock folded into their
// linear field) is assembled on the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "qb_internal.hpp"

struct qb_freeze {
    int32_t rounds = 0;
    std::vector<int32_t> kept;
    std::vector<double> d, w, field;
    std::vector<int32_t> row_ptr, ray, nbr_ptr, nbr;
    std::vector<float> a;
    double lambda = 0.0, kappa = 0.0;
};

namespace qb {
namespace {

// lb_i = sum_k w_b a_k (a_k / 2 - d_b) in the bit's CSR order, plus lin_i.
__global__ void freeze_bound_kernel(int n, const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ ray,
                                    const float* __restrict__ a, const double* __restrict__ w,
                                    const double* __restrict__ d, const double* __restrict__ field, double kappa,
                                    double* __restrict__ lb) {
    for (int i = int(blockIdx.x * blockDim.x + threadIdx.x); i < n; i += int(gridDim.x * blockDim.x)) {
        double acc = 0.0;
        for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
            const int b = ray[k];
            const double ak = double(a[k]);
            acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(w[b], ak), __dsub_rn(__dmul_rn(0.5, ak), d[b])));
        }
        lb[i] = __dadd_rn(acc, field ? field[i] : kappa);
    }
}

// One Jacobi round: a free bit freezes when its bound, with the neighbours
// frozen so far, reaches the margin.
__global__ void freeze_round_kernel(int n, const int32_t* __restrict__ nbr_ptr, const int32_t* __restrict__ nbr,
                                    const double* __restrict__ lb, double lambda, double margin,
                                    const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int* changed) {
    for (int i = int(blockIdx.x * blockDim.x + threadIdx.x); i < n; i += int(gridDim.x * blockDim.x)) {
        if (in[i]) {
            out[i] = 1;
            continue;
        }
        int rock = 0, free = 0;
        for (int k = nbr_ptr[i]; k < nbr_ptr[i + 1]; ++k) (in[nbr[k]] ? rock : free)++;
        const double bound = __dadd_rn(lb[i], __dmul_rn(lambda, double(rock - free)));
        const uint8_t f = bound >= margin ? 1 : 0;
        out[i] = f;
        if (f) *changed = 1;
    }
}

}  // namespace
}  // namespace qb

extern "C" qb_status qb_freeze_rock(const qb_residual_desc* desc, double margin, const qb_opts* opts,
                                    qb_freeze** out) {
    return qb::guarded("qb_freeze_rock", [&]() -> qb_status {
        using namespace qb;
        if (!desc || !out) return fail(QB_EINVAL, "qb_freeze_rock: null argument");
        *out = nullptr;
        if (!(desc->lambda >= 0.0)) return fail(QB_EINVAL, "qb_freeze_rock: needs lambda >= 0 (bounds must grow as bits freeze)");
        if (!std::isfinite(margin)) return fail(QB_EINVAL, "qb_freeze_rock: margin must be finite");
        const int n = desc->n_vars, nr = desc->n_rays;
        if (n <= 0 || nr < 0 || !desc->row_ptr || !desc->nbr_ptr || (nr > 0 && (!desc->d || !desc->w)))
            return fail(QB_EINVAL, "qb_freeze_rock: malformed problem");
        const int64_t nnz = desc->row_ptr[n], nn = desc->nbr_ptr[n];
        cudaStream_t st = opts ? static_cast<cudaStream_t>(opts->stream) : nullptr;
        if (opts && opts->device >= 0) QB_CUDA(cudaSetDevice(opts->device));
        DevBuf d_row, d_ray, d_a, d_w, d_d, d_field, d_nptr, d_nbr, d_lb, d_f0, d_f1, d_changed;
        qb_status s;
        if ((s = upload(d_row, desc->row_ptr, (size_t(n) + 1) * 4, st))) return s;
        if ((s = upload(d_ray, desc->ray, size_t(nnz) * 4, st))) return s;
        if ((s = upload(d_a, desc->a, size_t(nnz) * 4, st))) return s;
        if ((s = upload(d_w, desc->w, size_t(nr) * 8, st))) return s;
        if ((s = upload(d_d, desc->d, size_t(nr) * 8, st))) return s;
        if (desc->field && (s = upload(d_field, desc->field, size_t(n) * 8, st))) return s;
        if ((s = upload(d_nptr, desc->nbr_ptr, (size_t(n) + 1) * 4, st))) return s;
        if ((s = upload(d_nbr, desc->nbr, size_t(nn) * 4, st))) return s;
        if ((s = d_lb.alloc(size_t(n) * 8))) return s;
        if ((s = d_f0.alloc(size_t(n)))) return s;
        if ((s = d_f1.alloc(size_t(n)))) return s;
        if ((s = d_changed.alloc(sizeof(int)))) return s;
        QB_CUDA(cudaMemsetAsync(d_f0.p, 0, size_t(n), st));
        const int threads = 256;
        const int blocks = int(std::min<int64_t>((n + threads - 1) / threads, 148 * 16));
        freeze_bound_kernel<<<blocks, threads, 0, st>>>(n, d_row.as<int32_t>(), d_ray.as<int32_t>(), d_a.as<float>(),
                                                        d_w.as<double>(), d_d.as<double>(),
                                                        desc->field ? d_field.as<double>() : nullptr, desc->kappa,
                                                        d_lb.as<double>());
        QB_CUDA(cudaGetLastError());
        std::unique_ptr<qb_freeze> F(new (std::nothrow) qb_freeze());
        if (!F) return fail(QB_ENOMEM, "qb_freeze_rock: out of host memory");
        DevBuf* in = &d_f0;
        DevBuf* nx = &d_f1;
        for (;;) {
            int changed = 0;
            QB_CUDA(cudaMemsetAsync(d_changed.p, 0, sizeof(int), st));
            freeze_round_kernel<<<blocks, threads, 0, st>>>(n, d_nptr.as<int32_t>(), d_nbr.as<int32_t>(), d_lb.as<double>(),
                                                            desc->lambda, margin, in->as<uint8_t>(), nx->as<uint8_t>(),
                                                            d_changed.as<int>());
            QB_CUDA(cudaGetLastError());
            QB_CUDA(cudaMemcpyAsync(&changed, d_changed.p, sizeof(int), cudaMemcpyDeviceToHost, st));
            QB_CUDA(cudaStreamSynchronize(st));
            ++F->rounds;
            std::swap(in, nx);
            if (!changed) break;
        }
        std::vector<uint8_t> frozen(static_cast<size_t>(n));
        QB_CUDA(cudaMemcpy(frozen.data(), in->p, size_t(n), cudaMemcpyDeviceToHost));
        // the reduced problem: kept bits in order, bonds to frozen rock in the field
        std::vector<int32_t> new_index(static_cast<size_t>(n), -1);
        for (int i = 0; i < n; ++i)
            if (!frozen[size_t(i)]) {
                new_index[size_t(i)] = int32_t(F->kept.size());
                F->kept.push_back(i);
            }
        F->lambda = desc->lambda;
        F->kappa = desc->kappa;
        F->d.assign(desc->d, desc->d + nr);
        F->w.assign(desc->w, desc->w + nr);
        F->row_ptr.push_back(0);
        F->nbr_ptr.push_back(0);
        for (int i : F->kept) {
            for (int k = desc->row_ptr[i]; k < desc->row_ptr[i + 1]; ++k) {
                F->ray.push_back(desc->ray[k]);
                F->a.push_back(desc->a[k]);
            }
            F->row_ptr.push_back(int32_t(F->ray.size()));
            int rock = 0;
            for (int k = desc->nbr_ptr[i]; k < desc->nbr_ptr[i + 1]; ++k) {
                if (frozen[size_t(desc->nbr[k])]) ++rock;
                else F->nbr.push_back(new_index[size_t(desc->nbr[k])]);
            }
            F->nbr_ptr.push_back(int32_t(F->nbr.size()));
            const double lin = desc->field ? desc->field[i] : desc->kappa;
            F->field.push_back(lin + desc->lambda * double(rock));
        }
        *out = F.release();
        return QB_OK;
    });
}

extern "C" qb_status qb_freeze_info(const qb_freeze* f, int32_t* n_kept, int32_t* rounds) {
    if (!f) return qb::fail(QB_EINVAL, "qb_freeze_info: null handle");
    if (n_kept) *n_kept = int32_t(f->kept.size());
    if (rounds) *rounds = f->rounds;
    return QB_OK;
}

extern "C" qb_status qb_freeze_kept(const qb_freeze* f, int32_t* kept) {
    if (!f || (!kept && !f->kept.empty())) return qb::fail(QB_EINVAL, "qb_freeze_kept: null argument");
    if (!f->kept.empty()) std::memcpy(kept, f->kept.data(), f->kept.size() * 4);
    return QB_OK;
}

extern "C" qb_status qb_freeze_reduced(const qb_freeze* f, qb_residual_desc* r) {
    if (!f || !r) return qb::fail(QB_EINVAL, "qb_freeze_reduced: null argument");
    r->n_vars = int32_t(f->kept.size());
    r->n_rays = int32_t(f->d.size());
    r->d = f->d.data();
    r->w = f->w.data();
    r->row_ptr = f->row_ptr.data();
    r->ray = f->ray.data();
    r->a = f->a.data();
    r->nbr_ptr = f->nbr_ptr.data();
    r->nbr = f->nbr.data();
    r->lambda = f->lambda;
    r->kappa = f->kappa;
    r->field = f->field.data();
    return QB_OK;
}

extern "C" void qb_freeze_destroy(qb_freeze* f) { delete f; }
