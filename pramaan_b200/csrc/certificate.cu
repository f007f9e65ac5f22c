// certificate.cu — FP64 solution certificates of many LPs on the GPU.
//
// For each LP of a batch and each given point (x, y) it computes, in FP64:
//   * the reference certificate's quantities (src/certificate/certificate.cpp:
//     38-43 objective c^T x + offset in the model's sense, 45-62 the maximum
//     row violation, 64-79 the maximum variable-bound violation; integrality
//     is 0 for LPs), and
//   * the relative KKT error of (x, y) (PDLP definitions): the primal residual
//     ||(dist(Ax, [l_r, u_r]), dist(x, [l_x, u_x]))|| / (1 + ||b||), the dual
//     residual of the reduced cost rc = c + A^T y (the solver's y is the
//     negated multiplier) projected on the bound cone / (1 + ||c||), and the
//     gap |p - d| / (1 + |p| + |d|), with the problem in minimisation form.
// The LPs are packed block-diagonally once; every point costs two FP64
// products (A x, A^T y over the FP32 hi + lo split of the values, exact to
// about 2^-48 of each value), one contribution pass per side and a per-LP
// reduction in a fixed order, so results are deterministic.
#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include "certificate.cuh"

namespace pb {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 4096;
constexpr double kInf = 1e29;
// contribution slots per element: rows use 0-3 (rp2, b2, dobj, rd2), columns
// 0-5 (rp2, c2, pobj, dobj, rd2, model-sense objective); slot 7 is a maximum
// (row violation / bound violation), the others are sums
constexpr int kWidth = 8;

int grid(long long n) { return int(std::max<long long>(1, std::min<long long>((n + kThreads - 1) / kThreads, 148LL * 64))); }

#define CERT_STRIDE(i, n) \
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

// cold start x0 = clamp(0, l, u)
__global__ void cold_x_kernel(const double* __restrict__ lo, const double* __restrict__ hi, int n,
                              double* __restrict__ x) {
    CERT_STRIDE(j, n) {
        double v = 0.0;
        if (hi[j] < kInf && v > hi[j]) v = hi[j];
        if (lo[j] > -kInf && v < lo[j]) v = lo[j];
        x[j] = v;
    }
}

// rows: slots 0-3 sums (rp2, b2, dobj, rd2), slot 7 max row violation
__global__ void row_contrib_kernel(const double* __restrict__ act, const double* __restrict__ y,
                                   const double* __restrict__ lo, const double* __restrict__ hi, int m,
                                   double* __restrict__ out) {
    CERT_STRIDE(i, m) {
        const double a = act[i], l = lo[i], h = hi[i];
        double d = 0.0, viol = 0.0;
        if (l > -kInf && a < l) d = l - a;
        if (h < kInf && a > h) d = a - h;
        if (l > -kInf) viol = fmax(viol, l - a);
        if (h < kInf) viol = fmax(viol, a - h);
        double b2 = 0.0;
        if (l > -kInf) b2 += l * l;
        if (h < kInf && !(l > -kInf && l == h)) b2 += h * h;
        const double lam = -y[i];
        double dobj = 0.0, rd2 = 0.0;
        if (lam > 0.0) { if (l > -kInf) dobj = lam * l; else rd2 = lam * lam; }
        else if (lam < 0.0) { if (h < kInf) dobj = lam * h; else rd2 = lam * lam; }
        double* o = out + size_t(i) * kWidth;
        o[0] = d * d; o[1] = b2; o[2] = dobj; o[3] = rd2;
        o[4] = 0.0; o[5] = 0.0; o[6] = 0.0; o[7] = viol;
    }
}

// columns: slots 0-5 sums (rp2, c2, pobj, dobj, rd2, obj), slot 7 max bound violation
__global__ void col_contrib_kernel(const double* __restrict__ x, const double* __restrict__ aty,
                                   const double* __restrict__ cmin, const double* __restrict__ c_model,
                                   const double* __restrict__ lo, const double* __restrict__ hi, int n,
                                   double* __restrict__ out) {
    CERT_STRIDE(j, n) {
        const double xj = x[j], l = lo[j], h = hi[j], c = cmin[j];
        double v = 0.0, viol = 0.0;
        if (l > -kInf && xj < l) v = l - xj;
        if (h < kInf && xj > h) v = xj - h;
        if (l > -kInf) viol = fmax(viol, l - xj);
        if (h < kInf) viol = fmax(viol, xj - h);
        const double r = c + aty[j];
        double dobj = 0.0, rd2 = 0.0;
        if (r > 0.0) { if (l > -kInf) dobj = r * l; else rd2 = r * r; }
        else if (r < 0.0) { if (h < kInf) dobj = r * h; else rd2 = r * r; }
        double* o = out + size_t(j) * kWidth;
        o[0] = v * v; o[1] = c * c; o[2] = c * xj; o[3] = dobj; o[4] = rd2; o[5] = c_model[j] * xj;
        o[6] = 0.0; o[7] = viol;
    }
}

// One block per chunk; sums of slots 0-6, max of slot 7 (fixed tree order).
__global__ void chunk_kernel(const double* __restrict__ contrib, const int* __restrict__ begin,
                             double* __restrict__ out) {
    __shared__ double sh[kWidth][kThreads];
    const int c = blockIdx.x;
    const int b = begin[c], e = begin[c + 1];
    double acc[kWidth] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = b + threadIdx.x; i < e; i += blockDim.x)
#pragma unroll
        for (int s = 0; s < kWidth; ++s) {
            const double v = contrib[size_t(i) * kWidth + s];
            acc[s] = s == kWidth - 1 ? fmax(acc[s], v) : acc[s] + v;
        }
#pragma unroll
    for (int s = 0; s < kWidth; ++s) sh[s][threadIdx.x] = acc[s];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
#pragma unroll
            for (int s = 0; s < kWidth; ++s) {
                const double a = sh[s][threadIdx.x], o = sh[s][threadIdx.x + w];
                sh[s][threadIdx.x] = s == kWidth - 1 ? fmax(a, o) : a + o;
            }
        __syncthreads();
    }
    if (threadIdx.x < kWidth) out[size_t(c) * kWidth + threadIdx.x] = sh[threadIdx.x][0];
}

// One thread per (LP, slot): the LP's chunks in order.
__global__ void lp_kernel(const double* __restrict__ chunk_out, const int* __restrict__ lp_first, int K,
                          double* __restrict__ out) {
    CERT_STRIDE(t, (long long)K * kWidth) {
        const int k = int(t / kWidth), s = int(t % kWidth);
        double acc = 0.0;
        for (int c = lp_first[k]; c < lp_first[k + 1]; ++c) {
            const double v = chunk_out[size_t(c) * kWidth + s];
            acc = s == kWidth - 1 ? fmax(acc, v) : acc + v;
        }
        out[t] = acc;
    }
}

template <typename Epi>
void product(const CsrDevice& A, const double* x, const Epi& e, int* status, cudaStream_t st, int dev) {
    if (A.has_lo)
        SpmvLauncher<Epi, double, double, true>::launch(A.view(true), x, e, status, st, dev);
    else
        SpmvLauncher<Epi, double, double, false>::launch(A.view(false), x, e, status, st, dev);
}

void build_chunks(const std::vector<int>& seg, std::vector<int>& begin, std::vector<int>& first) {
    const int K = int(seg.size()) - 1;
    first.assign(size_t(K) + 1, 0);
    begin.clear();
    for (int k = 0; k < K; ++k) {
        first[size_t(k)] = int(begin.size());
        for (int b = seg[size_t(k)]; b < seg[size_t(k) + 1]; b += kChunk) begin.push_back(b);
    }
    first[size_t(K)] = int(begin.size());
    begin.push_back(seg[size_t(K)]);
}

}  // namespace

CertificateBatch::CertificateBatch(const pramaan_lp* lps, int count, int device) : dev_(device), count_(count) {
    long long M = 0, N = 0, NZ = 0;
    for (int k = 0; k < count; ++k) {
        const pramaan_lp& lp = lps[k];
        if (lp.num_rows < 0 || lp.num_cols < 0 || lp.nnz < 0) throw InvalidArgument("certificate: negative size");
        if (lp.num_cols > 0 && (!lp.obj_coeffs || !lp.var_lower || !lp.var_upper))
            throw InvalidArgument("certificate: column data is NULL");
        if (lp.num_rows > 0 && (!lp.row_ptr || !lp.row_lower || !lp.row_upper))
            throw InvalidArgument("certificate: row data is NULL");
        if (lp.nnz > 0 && (!lp.col_idx || !lp.values)) throw InvalidArgument("certificate: col_idx/values is NULL");
        r0_.push_back(int(M));
        c0_.push_back(int(N));
        M += lp.num_rows;
        N += lp.num_cols;
        NZ += lp.nnz;
        if (M > INT_MAX / 2 || N > INT_MAX / 2 || NZ > INT_MAX / 2)
            throw InvalidArgument("certificate: the packed batch exceeds 2^30 rows, columns or non-zeros");
    }
    r0_.push_back(int(M));
    c0_.push_back(int(N));
    m_ = int(M);
    n_ = int(N);
    nnz_ = int(NZ);
    PB_CUDA_CHECK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    status_.alloc(1);
    PB_CUDA_CHECK(cudaMemsetAsync(status_.get(), 0, 4, st_));
    const size_t Mz = size_t(m_), Nz = size_t(n_), Ez = size_t(nnz_);
    std::vector<int> rp(Mz + 1), ci(Ez);
    std::vector<double> val(Ez), rl(Mz), ru(Mz), vl(Nz), vu(Nz), cmin(Nz), cmod(Nz);
    offset_.resize(size_t(count));
    long long e0 = 0;
    for (int k = 0; k < count; ++k) {
        const pramaan_lp& lp = lps[k];
        const int R = r0_[size_t(k)], Cc = c0_[size_t(k)];
        const double sign = lp.obj_sense == PRAMAAN_MAXIMIZE ? -1.0 : 1.0;
        offset_[size_t(k)] = lp.obj_offset;
        if (lp.num_rows > 0 && (lp.row_ptr[0] != 0 || lp.row_ptr[lp.num_rows] != lp.nnz))
            throw InvalidArgument("pramaan_lp: row_ptr must start at 0, be non-decreasing and end at nnz");
        for (int i = 0; i < lp.num_rows; ++i) {
            rp[size_t(R + i)] = int(e0 + lp.row_ptr[i]);
            rl[size_t(R + i)] = lp.row_lower[i];
            ru[size_t(R + i)] = lp.row_upper[i];
        }
        for (int e = 0; e < lp.nnz; ++e) {
            const int j = lp.col_idx[e];
            if (j < 0 || j >= lp.num_cols) throw InvalidArgument("pramaan_lp: col_idx entry out of bounds");
            ci[size_t(e0 + e)] = Cc + j;
            val[size_t(e0 + e)] = lp.values[e];
        }
        for (int j = 0; j < lp.num_cols; ++j) {
            cmin[size_t(Cc + j)] = sign * lp.obj_coeffs[j];
            cmod[size_t(Cc + j)] = lp.obj_coeffs[j];
            vl[size_t(Cc + j)] = lp.var_lower[j];
            vu[size_t(Cc + j)] = lp.var_upper[j];
        }
        e0 += lp.nnz;
    }
    rp[Mz] = int(e0);
    DevBuf<int> flag(1);
    PB_CUDA_CHECK(cudaMemsetAsync(flag.get(), 0, 4, st_));
    csr_upload_f64(A_, m_, n_, nnz_, rp.data(), ci.data(), val.data(), st_, flag.get());
    int h_flag = 0;
    PB_CUDA_CHECK(cudaMemcpyAsync(&h_flag, flag.get(), 4, cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
    if (h_flag & 1) throw InvalidArgument("pramaan_lp: row_ptr must start at 0, be non-decreasing and end at nnz");
    if (h_flag & 2) throw InvalidArgument("pramaan_lp: col_idx entry out of bounds");
    csr_transpose(A_, AT_, st_);
    A_.pack(st_);
    AT_.pack(st_);
    SpmvLauncher<EpiStore<double, double>, double, double, true>::blocks_per_sm(dev_);
    SpmvLauncher<EpiStore<double, double>, double, double, false>::blocks_per_sm(dev_);
    auto up = [&](auto& d, const auto& h) {
        d.alloc(h.size());
        if (!h.empty())
            PB_CUDA_CHECK(cudaMemcpyAsync(d.get(), h.data(), h.size() * sizeof(h[0]), cudaMemcpyHostToDevice, st_));
    };
    up(rlo_, rl); up(rhi_, ru); up(vlo_, vl); up(vhi_, vu); up(cmin_, cmin); up(cmod_, cmod);
    std::vector<int> rb, rf, cb, cf;
    build_chunks(r0_, rb, rf);
    build_chunks(c0_, cb, cf);
    rchunks_ = int(rb.size()) - 1;
    cchunks_ = int(cb.size()) - 1;
    up(rbegin_, rb); up(rfirst_, rf); up(cbegin_, cb); up(cfirst_, cf);
    x_.alloc(Nz > 0 ? Nz : 1);
    y_.alloc(Mz > 0 ? Mz : 1);
    act_.alloc(Mz > 0 ? Mz : 1);
    aty_.alloc(Nz > 0 ? Nz : 1);
    contrib_.alloc(std::max(Mz, Nz) * kWidth + kWidth);
    chunk_out_.alloc(size_t(std::max(rchunks_, cchunks_) + 1) * kWidth);
    lp_out_.alloc(size_t(std::max(count, 1)) * kWidth * 2);
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
}

CertificateBatch::~CertificateBatch() {
    if (st_) {
        cudaStreamSynchronize(st_);
        cudaStreamDestroy(st_);
    }
}

void CertificateBatch::evaluate(const pramaan_warm_start* points, pramaan_certificate* out) {
    const int K = count_;
    if (K == 0) return;
    // gather the point into the packed layout (x NULL: the cold start; y NULL: 0)
    std::vector<double> hx(size_t(n_), 0.0), hy(size_t(m_), 0.0);
    std::vector<char> cold(size_t(K), 0);
    for (int k = 0; k < K; ++k) {
        const pramaan_warm_start& p = points[k];
        const int nk = c0_[size_t(k) + 1] - c0_[size_t(k)], mk = r0_[size_t(k) + 1] - r0_[size_t(k)];
        if (p.x)
            for (int j = 0; j < nk; ++j) hx[size_t(c0_[size_t(k)] + j)] = p.x[j];
        else
            cold[size_t(k)] = 1;
        if (p.y)
            for (int i = 0; i < mk; ++i) hy[size_t(r0_[size_t(k)] + i)] = p.y[i];
    }
    if (n_ > 0) PB_CUDA_CHECK(cudaMemcpyAsync(x_.get(), hx.data(), size_t(n_) * 8, cudaMemcpyHostToDevice, st_));
    if (m_ > 0) PB_CUDA_CHECK(cudaMemcpyAsync(y_.get(), hy.data(), size_t(m_) * 8, cudaMemcpyHostToDevice, st_));
    // cold-start LPs: x0 = clamp(0, l, u) over their columns
    for (int k = 0; k < K; ++k) {
        if (!cold[size_t(k)]) continue;
        const int C = c0_[size_t(k)], nk = c0_[size_t(k) + 1] - C;
        if (nk > 0)
            cold_x_kernel<<<grid(nk), kThreads, 0, st_>>>(vlo_.get() + C, vhi_.get() + C, nk, x_.get() + C);
    }
    PB_CUDA_CHECK(cudaGetLastError());
    if (m_ > 0) {
        product(A_, x_.get(), EpiStore<double, double>{act_.get()}, status_.get(), st_, dev_);
        row_contrib_kernel<<<grid(m_), kThreads, 0, st_>>>(act_.get(), y_.get(), rlo_.get(), rhi_.get(), m_,
                                                           contrib_.get());
        chunk_kernel<<<rchunks_ > 0 ? rchunks_ : 1, kThreads, 0, st_>>>(contrib_.get(), rbegin_.get(), chunk_out_.get());
        lp_kernel<<<grid((long long)K * kWidth), kThreads, 0, st_>>>(chunk_out_.get(), rfirst_.get(), K, lp_out_.get());
        product(AT_, y_.get(), EpiStore<double, double>{aty_.get()}, status_.get(), st_, dev_);
    } else {
        PB_CUDA_CHECK(cudaMemsetAsync(lp_out_.get(), 0, size_t(K) * kWidth * 8, st_));
    }
    if (n_ > 0) {
        if (m_ == 0) PB_CUDA_CHECK(cudaMemsetAsync(aty_.get(), 0, size_t(n_) * 8, st_));
        col_contrib_kernel<<<grid(n_), kThreads, 0, st_>>>(x_.get(), aty_.get(), cmin_.get(), cmod_.get(),
                                                           vlo_.get(), vhi_.get(), n_, contrib_.get());
        chunk_kernel<<<cchunks_ > 0 ? cchunks_ : 1, kThreads, 0, st_>>>(contrib_.get(), cbegin_.get(), chunk_out_.get());
        lp_kernel<<<grid((long long)K * kWidth), kThreads, 0, st_>>>(chunk_out_.get(), cfirst_.get(), K,
                                                                     lp_out_.get() + size_t(K) * kWidth);
    } else {
        PB_CUDA_CHECK(cudaMemsetAsync(lp_out_.get() + size_t(K) * kWidth, 0, size_t(K) * kWidth * 8, st_));
    }
    PB_CUDA_CHECK(cudaGetLastError());
    std::vector<double> h(size_t(K) * kWidth * 2);
    PB_CUDA_CHECK(cudaMemcpyAsync(h.data(), lp_out_.get(), h.size() * 8, cudaMemcpyDeviceToHost, st_));
    int hs = 0;
    PB_CUDA_CHECK(cudaMemcpyAsync(&hs, status_.get(), 4, cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
    if (hs & kDevErrTimeout) throw DeviceTimeout("certificate: a TMA wait in a product exceeded its time limit");
    for (int k = 0; k < K; ++k) {
        const double* r = &h[size_t(k) * kWidth];
        const double* c = &h[size_t(K + k) * kWidth];
        pramaan_certificate& o = out[k];
        const double rp2 = r[0] + c[0], b2 = r[1], c2 = c[1], pobj = c[2], dobj = r[2] + c[3], rd2 = r[3] + c[4];
        o.objective_value = offset_[size_t(k)] + c[5];
        o.primal_residual = r[7];
        o.bound_violation = c[7];
        o.rel_primal = std::sqrt(rp2) / (1.0 + std::sqrt(b2));
        o.rel_dual = std::sqrt(rd2) / (1.0 + std::sqrt(c2));
        o.rel_gap = std::fabs(pobj - dobj) / (1.0 + std::fabs(pobj) + std::fabs(dobj));
        o.primal_objective = pobj;
        o.dual_objective = dobj;
        o.kkt = std::max(o.rel_primal, std::max(o.rel_dual, o.rel_gap));
    }
}

}  // namespace pb
