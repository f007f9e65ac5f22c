// panel.cu — the panel kernel, its launch, and the builder of the panel split
// (format and reasoning in panel.cuh).
#include "panel.cuh"

#include <algorithm>
#include <climits>
#include <cmath>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

namespace pb {

namespace {

constexpr int kThreads = 256;
inline int grid_for_n(long long n, int cap = 65535 * 8) {
    long long g = (n + kThreads - 1) / kThreads;
    if (g < 1) g = 1;
    return int(g < cap ? g : cap);
}

// ---------------------------------------------------------------------------
// The panel kernel
// ---------------------------------------------------------------------------

// Block p streams panel p's chunk records through per-warp rings (bulk copies
// completing on mbarriers, bounded waits) and writes part[p * L + r] for every
// long row r.
__global__ void __launch_bounds__(kPanelWarps * 32, 1)
    panel_product_kernel(const PanelView P, const float* __restrict__ x, int* __restrict__ dev_status) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int STAGES = kPanelStages;
    constexpr unsigned kBytes = unsigned(PanelRec::bytes);
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int p = blockIdx.x;
    // chunk_ptr and the records are written only when the operand is built,
    // so they may be read before the grid dependency wait.
    const int c0 = P.chunk_ptr[p];
    const int nch = P.chunk_ptr[p + 1] - c0;
    const int mine = warp < nch ? (nch - warp + kPanelWarps - 1) / kPanelWarps : 0;
    unsigned char* ring = smem + size_t(warp) * STAGES * PanelRec::bytes;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + PanelSmem::off_bar) + warp * STAGES;
    float* xs = reinterpret_cast<float*>(smem + PanelSmem::off_x);

    uint64_t policy = 0;
    auto issue = [&](int i) {
        const int c = c0 + warp + i * kPanelWarps;
        const int s = i % STAGES;
        mbar_arrive_expect_tx(&bar[s], kBytes);
        tma_bulk_g2s(ring + size_t(s) * PanelRec::bytes, P.rec + size_t(c) * PanelRec::bytes, kBytes, &bar[s],
                     policy);
    };
    // The ring holds only STAGES records per warp, too few bytes in flight to
    // cover HBM latency at full bandwidth: each warp also keeps its next
    // kPanelPrefetch records on their way into L2.
    auto prefetch = [&](int i) {
        if (i < mine) bulk_prefetch_l2(P.rec + size_t(c0 + warp + i * kPanelWarps) * PanelRec::bytes, kBytes);
    };
    if (lane == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(&bar[s], 1);
        fence_mbar_init();
        policy = l2_policy_evict_first();
        const int pre = mine < STAGES ? mine : STAGES;
        for (int i = 0; i < pre; ++i) issue(i);
        for (int i = STAGES; i < STAGES + kPanelPrefetch; ++i) prefetch(i);
    }
    __syncwarp();
    grid_dep_launch();
    grid_dep_wait();

    // Every thread issues kLoadBatch loads before it stores any, so a block's
    // start costs a few L2 round trips rather than one per loop pass.
    constexpr int kLoadBatch = 8;
    const int nthr = blockDim.x;
    if (P.vec_idx) {
        // ---- the gathered entries of x (the same for every block) ----
        const int V = P.vec_len;
        for (int k0 = threadIdx.x; k0 < V; k0 += nthr * kLoadBatch) {
            int idx[kLoadBatch];
            float v[kLoadBatch];
#pragma unroll
            for (int u = 0; u < kLoadBatch; ++u) {
                const int k = k0 + u * nthr;
                idx[u] = k < V ? __ldg(P.vec_idx + k) : 0;
            }
#pragma unroll
            for (int u = 0; u < kLoadBatch; ++u) v[u] = k0 + u * nthr < V ? __ldcg(x + idx[u]) : 0.f;
#pragma unroll
            for (int u = 0; u < kLoadBatch; ++u)
                if (k0 + u * nthr < V) xs[k0 + u * nthr] = v[u];
        }
    } else {
        // ---- panel p of x (W is a multiple of 4, x 16-byte aligned) ----
        const int col0 = p * P.width;
        int w = P.cols - col0;
        w = w < 0 ? 0 : (w > P.width ? P.width : w);
        const int w4 = w >> 2;
        const float4* x4 = reinterpret_cast<const float4*>(x + col0);
        float4* xs4 = reinterpret_cast<float4*>(xs);
        for (int k0 = threadIdx.x; k0 < w4; k0 += nthr * kLoadBatch) {
            float4 v[kLoadBatch];
#pragma unroll
            for (int u = 0; u < kLoadBatch; ++u)
                v[u] = k0 + u * nthr < w4 ? __ldcg(x4 + k0 + u * nthr) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int u = 0; u < kLoadBatch; ++u)
                if (k0 + u * nthr < w4) xs4[k0 + u * nthr] = v[u];
        }
        for (int k = (w4 << 2) + threadIdx.x; k < w; k += nthr) xs[k] = __ldcg(x + col0 + k);
    }
    __syncthreads();

    float* out_panel = P.part + size_t(p) * size_t(P.out_stride);
    bool failed = false;
    int i = 0;
    for (; i < mine; ++i) {
        const int s = i % STAGES;
        const uint32_t parity = uint32_t(i / STAGES) & 1u;
        const bool ok = mbar_wait_bounded_sleep(&bar[s], parity);
        if (__any_sync(0xffffffffu, !ok)) {
            failed = true;
            break;
        }
        unsigned char* st = ring + size_t(s) * PanelRec::bytes;
        const uint4* c16 = reinterpret_cast<const uint4*>(st + PanelRec::off_col);
        const float4* v4 = reinterpret_cast<const float4*>(st + PanelRec::off_val);
        const uint32_t* bits = reinterpret_cast<const uint32_t*>(st + PanelRec::off_bits);
        const int4 head = *reinterpret_cast<const int4*>(st + PanelRec::off_head);

        // ---- my 8 entries: columns, values, gathers from the panel ----
        // (the records are checked when built: every column lies in its panel)
        constexpr int IPT = kPanelIpt;
        float xv[IPT], vv[IPT];
        {
            const uint4 cc = c16[lane];
            const uint32_t wd[4] = {cc.x, cc.y, cc.z, cc.w};
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                xv[2 * t] = xs[wd[t] & 0xffffu];
                xv[2 * t + 1] = xs[wd[t] >> 16];
            }
        }
#pragma unroll
        for (int k = 0; k < IPT / 4; ++k) {
            const float4 v = v4[k * 32 + lane];
            vv[4 * k] = v.x; vv[4 * k + 1] = v.y; vv[4 * k + 2] = v.z; vv[4 * k + 3] = v.w;
        }
        const uint32_t my = (bits[lane >> 2] >> ((lane & 3) * 8)) & 0xffu;

        // ---- in-lane segmented prefix: pre[j] sums my entries from the last
        // segment start (or my first entry) through j, FMAs in entry order ----
        float pre[IPT];
        float acc = 0.f;
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            acc = __fmaf_rn(vv[j], xv[j], ((my >> j) & 1u) ? 0.f : acc);
            pre[j] = acc;
        }
        __syncwarp();   // every lane holds its values: the value slots take the prefixes
        float4* pre4 = reinterpret_cast<float4*>(st + PanelRec::off_val);   // panel_val_slot order
#pragma unroll
        for (int k = 0; k < IPT / 4; ++k)
            pre4[k * 32 + lane] = make_float4(pre[4 * k], pre[4 * k + 1], pre[4 * k + 2], pre[4 * k + 3]);
        __syncwarp();
        const float* pf = reinterpret_cast<const float*>(st + PanelRec::off_val);

        // ---- segments [a, b): one piece per lane they touch, each the prefix
        // at the piece's last entry, added in entry order ----
        const uint16_t* so = reinterpret_cast<const uint16_t*>(st + PanelRec::off_seg);
        float* out = out_panel + head.x;
        for (int sg = lane; sg < head.y; sg += 32) {
            const int a = so[sg], b = so[sg + 1];
            float sum = 0.f;
            if (a < b) {
                int e = (a | (IPT - 1)) + 1;
                e = e < b ? e : b;
                sum = pf[panel_val_slot(e - 1)];
                for (; e < b; e += IPT) sum += pf[panel_val_slot((e + IPT < b ? e + IPT : b) - 1)];
            }
            out[sg] = sum;
        }
        __syncwarp();   // stage s is free for the next copy
        if (lane == 0 && i + STAGES < mine) {
            fence_proxy_async_smem();
            issue(i + STAGES);
            prefetch(i + STAGES + kPanelPrefetch);
        }
    }
    if (failed && lane == 0) {
        atomicOr(dev_status, kDevErrTimeout);
        // Let every bulk copy this warp issued land before it retires.
        const int hi = (i + STAGES) < mine ? (i + STAGES) : mine;
        for (int j = i; j < hi; ++j) (void)mbar_wait_bounded(&bar[j % STAGES], uint32_t(j / STAGES) & 1u);
    }
    __syncwarp();
}


// ---------------------------------------------------------------------------
// Builder kernels
// ---------------------------------------------------------------------------

// Per row (and a trailing 0 at index rows, so exclusive scans end in totals):
// is_long, short length, long length.
__global__ void classify_rows_kernel(const int* __restrict__ rp, int rows, int thr, int* __restrict__ is_long,
                                     int* __restrict__ short_len, int* __restrict__ long_len) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= rows; i += gridDim.x * blockDim.x) {
        const int len = i < rows ? rp[i + 1] - rp[i] : 0;
        const bool lg = i < rows && len >= thr;
        is_long[i] = lg ? 1 : 0;
        short_len[i] = lg ? 0 : len;
        long_len[i] = lg ? len : 0;
    }
}

__global__ void long_row_list_kernel(const int* __restrict__ is_long, const int* __restrict__ lr_idx, int rows,
                                     int* __restrict__ long_row) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x)
        if (is_long[i]) long_row[lr_idx[i]] = i;
}

// The short rows' entries into the short operand (thread per row; short rows
// have fewer than `thr` entries).
__global__ void short_copy_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                  const float* __restrict__ val, const int* __restrict__ is_long, int rows,
                                  const int* __restrict__ s_rp, int* __restrict__ s_col, float* __restrict__ s_val) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        if (is_long[i]) continue;
        const int a = rp[i], b = rp[i + 1], d = s_rp[i];
        for (int k = a; k < b; ++k) {
            s_col[d + k - a] = col[k];
            s_val[d + k - a] = val[k];
        }
    }
}

// Rows of the short operand that are empty in A too (its other empty rows are
// the long rows, which the short product must leave alone).
__global__ void empty_in_a_kernel(const int* __restrict__ rp, const int* __restrict__ empty_rows, int k,
                                  char* __restrict__ keep) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
        const int r = empty_rows[i];
        keep[i] = rp[r + 1] == rp[r] ? 1 : 0;
    }
}

// The long rows' entries with their panel (the sort key), panel-local column,
// value and long-row index; one warp per row.
__global__ void long_entries_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                    const float* __restrict__ val, const int* __restrict__ is_long,
                                    const int* __restrict__ lr_idx, const int* __restrict__ l_off, int rows,
                                    int width, int* __restrict__ key, unsigned short* __restrict__ lcol,
                                    float* __restrict__ lval, int* __restrict__ lrow) {
    const int lane = threadIdx.x & 31;
    const long long w0 = (long long)(blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = (long long)(gridDim.x * blockDim.x) >> 5;
    for (long long i = w0; i < rows; i += nw) {
        if (!is_long[i]) continue;
        const int a = rp[i], b = rp[i + 1], o = l_off[i], r = lr_idx[i];
        for (int k = a + lane; k < b; k += 32) {
            const int c = col[k];
            const int p = c / width;
            const int pos = o + (k - a);
            key[pos] = p;
            lcol[pos] = static_cast<unsigned short>(c - p * width);
            lval[pos] = val[k];
            lrow[pos] = r;
        }
    }
}

__global__ void iota_kernel(int* __restrict__ a, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[i] = int(i);
}

// Entries per segment (p, r) and the longest segment.
__global__ void segment_count_kernel(const int* __restrict__ key, const int* __restrict__ lrow, long long nl,
                                     int L, int* __restrict__ cnt, int* __restrict__ longest) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nl; i += (long long)gridDim.x * blockDim.x) {
        const int c = atomicAdd(&cnt[(long long)key[i] * L + lrow[i]], 1) + 1;
        atomicMax(longest, c);
    }
}

// Greedy chunking of one panel's segments (thread per panel): a chunk closes
// before the segment that would take it past kPanelEnt entries or when it
// holds kPanelSegCap segments.  Pass 1 (desc == nullptr) counts the chunks
// into nch[p]; pass 2 writes {first segment, segments, first entry, panel}.
__global__ void chunk_kernel(const int* __restrict__ cnt, const int* __restrict__ segstart, int L, int P,
                             int* __restrict__ nch, const int* __restrict__ chunk_ptr, int4* __restrict__ desc) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const int* c = cnt + (long long)p * L;
    int k = 0, out = desc ? chunk_ptr[p] : 0;
    int r = 0;
    while (r < L) {
        const int first = r;
        int ent = 0;
        while (r < L && r - first < kPanelSegCap && ent + c[r] <= kPanelEnt) {
            ent += c[r];
            ++r;
        }
        if (desc) desc[out + k] = make_int4(first, r - first, segstart[(long long)p * L + first], p);
        ++k;
    }
    if (!desc) nch[p] = k;
}

// One block per chunk record.
__global__ void __launch_bounds__(256) fill_kernel(const int4* __restrict__ desc, int nchunks,
                                                   const int* __restrict__ cnt, const int* __restrict__ segstart,
                                                   int L, const int* __restrict__ perm,
                                                   const unsigned short* __restrict__ lcol,
                                                   const float* __restrict__ lval, unsigned char* __restrict__ rec) {
    __shared__ uint32_t bits[kPanelEnt / 32];
    for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const int4 d = desc[c];   // {first, nseg, entry base, panel}
        const long long sbase = (long long)d.w * L + d.x;
        const int nent = segstart[sbase + d.y] - d.z;
        unsigned char* R = rec + size_t(c) * PanelRec::bytes;
        if (threadIdx.x < kPanelEnt / 32) bits[threadIdx.x] = 0u;
        __syncthreads();
        uint16_t* so = reinterpret_cast<uint16_t*>(R + PanelRec::off_seg);
        for (int s = threadIdx.x; s <= d.y; s += blockDim.x) {
            const int off = segstart[sbase + s] - d.z;
            so[s] = static_cast<uint16_t>(off);
            if (s < d.y && cnt[sbase + s] > 0) atomicOr(&bits[off >> 5], 1u << (off & 31));
        }
        if (threadIdx.x == 0 && nent < kPanelEnt) atomicOr(&bits[nent >> 5], 1u << (nent & 31));
        uint16_t* cs = reinterpret_cast<uint16_t*>(R + PanelRec::off_col);
        float* vs = reinterpret_cast<float*>(R + PanelRec::off_val);
        for (int q = threadIdx.x; q < kPanelEnt; q += blockDim.x) {
            unsigned short cc = 0;
            float vv = 0.f;
            if (q < nent) {
                const int src = perm ? perm[d.z + q] : d.z + q;
                cc = lcol[src];
                vv = lval[src];
            }
            cs[panel_col_slot(q)] = cc;
            vs[panel_val_slot(q)] = vv;
        }
        __syncthreads();
        if (threadIdx.x < kPanelEnt / 32)
            reinterpret_cast<uint32_t*>(R + PanelRec::off_bits)[threadIdx.x] = bits[threadIdx.x];
        if (threadIdx.x == 0) *reinterpret_cast<int4*>(R + PanelRec::off_head) = make_int4(d.x, d.y, nent, 0);
        __syncthreads();
    }
}

// Checks every record once after it is built, so that the panel kernel can
// trust them without per-access clamps: segment count and offsets within the
// record, its segments within the long rows, every column inside its panel.
// vec_len > 0: every gather index must lie below vec_len (hot part of Aᵀy);
// else inside the record's panel of the columns.
__global__ void __launch_bounds__(256) check_records_kernel(const unsigned char* __restrict__ rec,
                                                            const int4* __restrict__ desc, int nchunks, int L,
                                                            int width, int cols, int vec_len,
                                                            int* __restrict__ bad) {
    for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const unsigned char* R = rec + size_t(c) * PanelRec::bytes;
        const int4 h = *reinterpret_cast<const int4*>(R + PanelRec::off_head);
        const int p = desc[c].w;
        int w = cols - p * width;
        w = w > width ? width : w;
        if (vec_len > 0) w = vec_len;
        const bool head_ok = h.y >= 0 && h.y <= kPanelSegCap && h.x >= 0 && h.x + h.y <= L && w > 0;
        if (!head_ok) {
            if (threadIdx.x == 0) atomicOr(bad, 1);
            continue;
        }
        const uint16_t* so = reinterpret_cast<const uint16_t*>(R + PanelRec::off_seg);
        const int nent = so[h.y];
        bool ok = nent <= kPanelEnt && nent == h.z;
        for (int s = threadIdx.x; s < h.y; s += blockDim.x) ok = ok && so[s] <= so[s + 1];
        const uint16_t* cs = reinterpret_cast<const uint16_t*>(R + PanelRec::off_col);
        for (int q = threadIdx.x; q < kPanelEnt; q += blockDim.x) ok = ok && int(cs[panel_col_slot(q)]) < w;
        if (!ok) atomicOr(bad, 1);
    }
}

template <typename T>
T read_one(const T* d, cudaStream_t st) {
    T h{};
    PB_CUDA_CHECK(cudaMemcpyAsync(&h, d, sizeof(T), cudaMemcpyDeviceToHost, st));
    PB_CUDA_CHECK(cudaStreamSynchronize(st));
    return h;
}

template <typename T>
void exclusive_sum(const T* in, T* out, long long n, cudaStream_t st) {
    size_t tb = 0;
    PB_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, n, st));
    DevBuf<unsigned char> temp(tb > 0 ? tb : 1);
    PB_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(temp.get(), tb, in, out, n, st));
    PB_CUDA_CHECK(cudaStreamSynchronize(st));   // temp is freed on return
}

}  // namespace

// Shared memory one panel block may use on `dev` (the opt-in maximum, at most
// PanelSmem::max_bytes).
static size_t panel_smem_limit(int dev) {
    int optin = 0;
    PB_CUDA_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    return std::min(size_t(optin > 0 ? optin : 0), PanelSmem::max_bytes);
}

void panel_prepare(int dev) {
    PB_CUDA_CHECK(cudaFuncSetAttribute(&panel_product_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(panel_smem_limit(dev))));
}

void panel_product_launch(const PanelView& v, const float* x, int* dev_status, cudaStream_t st) {
    if (v.panels <= 0 || v.out_stride <= 0) return;
    launch_dependent(&panel_product_kernel, v.panels, kPanelWarps * 32,
                     PanelSmem::bytes(v.vec_idx ? v.vec_len : v.width), st, v, x, dev_status);
}

void build_panel_split(const CsrDevice& A, PanelSplit& ps, int mode, int dev, cudaStream_t st) {
    ps = PanelSplit{};
    const int rows = A.rows, cols = A.cols;
    const long long nnz = A.nnz;
    if (mode < 0 || rows <= 0 || cols <= 0 || nnz <= 0) return;
    if (A.packed || !A.col.get() || !A.val.get()) throw std::logic_error("build_panel_split needs the flat operand");
    if (mode == 0 && nnz < kPanelMinNnz) return;
    const int sms = device_sm_count(dev);
    int width = (cols + sms - 1) / sms;
    width = (width + 3) / 4 * 4;
    const size_t limit = panel_smem_limit(dev);
    if (limit <= PanelSmem::off_x || PanelSmem::bytes(width) > limit || width > 65536) return;
    const int panels = (cols + width - 1) / width;
    const int thr = mode >= 2 ? mode : std::max(2, int(std::ceil(kPanelLenPerPanel * panels)));

    // ---- classify the rows ----
    DevBuf<int> is_long{size_t(rows) + 1}, slen{size_t(rows) + 1}, llen{size_t(rows) + 1};
    DevBuf<int> lr_idx{size_t(rows) + 1}, s_rp{size_t(rows) + 1}, l_off{size_t(rows) + 1};
    classify_rows_kernel<<<grid_for_n(rows + 1LL), kThreads, 0, st>>>(A.row_ptr.get(), rows, thr, is_long.get(),
                                                                       slen.get(), llen.get());
    PB_CUDA_CHECK(cudaGetLastError());
    exclusive_sum(is_long.get(), lr_idx.get(), rows + 1LL, st);
    exclusive_sum(slen.get(), s_rp.get(), rows + 1LL, st);
    exclusive_sum(llen.get(), l_off.get(), rows + 1LL, st);
    const int L = read_one(lr_idx.get() + rows, st);
    const int ns = read_one(s_rp.get() + rows, st);
    const long long nl = read_one(l_off.get() + rows, st);
    if (L <= 0) return;
    if (mode == 0 && double(nl) < kPanelMinShare * double(nnz)) return;
    if ((long long)panels * L + 1 > INT_MAX) return;

    // ---- segments: panel and long row of every long entry, counts ----
    DevBuf<int> key{size_t(nl)}, lrow{size_t(nl)};
    DevBuf<unsigned short> lcol{size_t(nl)};
    DevBuf<float> lval{size_t(nl)};
    long_entries_kernel<<<grid_for_n((long long)rows * 32), kThreads, 0, st>>>(
        A.row_ptr.get(), A.col.get(), A.val.get(), is_long.get(), lr_idx.get(), l_off.get(), rows, width, key.get(),
        lcol.get(), lval.get(), lrow.get());
    PB_CUDA_CHECK(cudaGetLastError());
    const long long nseg = (long long)panels * L;
    DevBuf<int> cnt{size_t(nseg) + 1}, segstart{size_t(nseg) + 1}, longest(1);
    PB_CUDA_CHECK(cudaMemsetAsync(cnt.get(), 0, cnt.bytes(), st));
    PB_CUDA_CHECK(cudaMemsetAsync(longest.get(), 0, 4, st));
    segment_count_kernel<<<grid_for_n(nl), kThreads, 0, st>>>(key.get(), lrow.get(), nl, L, cnt.get(),
                                                               longest.get());
    PB_CUDA_CHECK(cudaGetLastError());
    if (read_one(longest.get(), st) > kPanelEnt) return;   // a segment longer than a chunk
    lrow.reset();
    exclusive_sum(cnt.get(), segstart.get(), nseg + 1, st);

    // ---- entries in panel order (stable: long row, then CSR order, within a panel) ----
    DevBuf<int> perm{size_t(nl)};
    {
        DevBuf<int> key_out{size_t(nl)}, iota{size_t(nl)};
        iota_kernel<<<grid_for_n(nl), kThreads, 0, st>>>(iota.get(), nl);
        PB_CUDA_CHECK(cudaGetLastError());
        int end_bit = 1;
        while ((1 << end_bit) < panels) ++end_bit;
        size_t tb = 0;
        PB_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, tb, key.get(), key_out.get(), iota.get(), perm.get(),
                                                      nl, 0, end_bit, st));
        DevBuf<unsigned char> temp(tb > 0 ? tb : 1);
        PB_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(temp.get(), tb, key.get(), key_out.get(), iota.get(),
                                                      perm.get(), nl, 0, end_bit, st));
        PB_CUDA_CHECK(cudaStreamSynchronize(st));
    }
    key.reset();

    // ---- chunks ----
    DevBuf<int> nch{size_t(panels) + 1};
    PB_CUDA_CHECK(cudaMemsetAsync(nch.get(), 0, nch.bytes(), st));
    chunk_kernel<<<(panels + 63) / 64, 64, 0, st>>>(cnt.get(), segstart.get(), L, panels, nch.get(), nullptr,
                                                    nullptr);
    PB_CUDA_CHECK(cudaGetLastError());
    ps.chunk_ptr.alloc(size_t(panels) + 1);
    exclusive_sum(nch.get(), ps.chunk_ptr.get(), panels + 1LL, st);
    const int nchunks = read_one(ps.chunk_ptr.get() + panels, st);
    DevBuf<int4> desc{size_t(nchunks > 0 ? nchunks : 1)};
    chunk_kernel<<<(panels + 63) / 64, 64, 0, st>>>(cnt.get(), segstart.get(), L, panels, nullptr,
                                                    ps.chunk_ptr.get(), desc.get());
    PB_CUDA_CHECK(cudaGetLastError());
    ps.rec.alloc(size_t(nchunks) * PanelRec::bytes);
    PB_CUDA_CHECK(cudaMemsetAsync(ps.rec.get(), 0, ps.rec.bytes(), st));
    fill_kernel<<<std::min(nchunks, 65535 * 8), 256, 0, st>>>(desc.get(), nchunks, cnt.get(), segstart.get(), L,
                                                             perm.get(), lcol.get(), lval.get(), ps.rec.get());
    PB_CUDA_CHECK(cudaGetLastError());
    {
        DevBuf<int> bad(1);
        PB_CUDA_CHECK(cudaMemsetAsync(bad.get(), 0, 4, st));
        check_records_kernel<<<std::min(nchunks, 65535 * 8), 256, 0, st>>>(ps.rec.get(), desc.get(), nchunks, L,
                                                                          width, cols, 0, bad.get());
        PB_CUDA_CHECK(cudaGetLastError());
        if (read_one(bad.get(), st)) throw std::logic_error("build_panel_split: a panel record failed its check");
    }
    ps.long_row.alloc(size_t(L));
    long_row_list_kernel<<<grid_for_n(rows), kThreads, 0, st>>>(is_long.get(), lr_idx.get(), rows,
                                                                 ps.long_row.get());
    PB_CUDA_CHECK(cudaGetLastError());
    ps.part.alloc(size_t(nseg));

    // ---- the short rows as their own operand ----
    CsrDevice& S = ps.S;
    S.allocate(rows, cols, ns, /*lo=*/false);
    PB_CUDA_CHECK(cudaMemcpyAsync(S.row_ptr.get(), s_rp.get(), (size_t(rows) + 1) * 4, cudaMemcpyDeviceToDevice, st));
    if (ns > 0) {
        short_copy_kernel<<<grid_for_n(rows), kThreads, 0, st>>>(A.row_ptr.get(), A.col.get(), A.val.get(),
                                                                 is_long.get(), rows, s_rp.get(), S.col.get(),
                                                                 S.val.get());
        PB_CUDA_CHECK(cudaGetLastError());
    }
    S.finalize(st);
    if (S.num_empty > 0) {
        // keep only the rows that are empty in A: the fixup writes those as 0
        const int k = S.num_empty;
        DevBuf<char> keep{size_t(k)};
        DevBuf<int> kept{size_t(k)}, nkept(1);
        empty_in_a_kernel<<<grid_for_n(k), kThreads, 0, st>>>(A.row_ptr.get(), S.empty_rows.get(), k, keep.get());
        PB_CUDA_CHECK(cudaGetLastError());
        size_t tb = 0;
        PB_CUDA_CHECK(cub::DeviceSelect::Flagged(nullptr, tb, S.empty_rows.get(), keep.get(), kept.get(),
                                                 nkept.get(), k, st));
        DevBuf<unsigned char> temp(tb > 0 ? tb : 1);
        PB_CUDA_CHECK(cub::DeviceSelect::Flagged(temp.get(), tb, S.empty_rows.get(), keep.get(), kept.get(),
                                                 nkept.get(), k, st));
        S.num_empty = read_one(nkept.get(), st);
        S.empty_rows = std::move(kept);
    }
    S.pack(st);
    PB_CUDA_CHECK(cudaStreamSynchronize(st));   // temporaries are freed on return

    ps.active = true;
    ps.panels = panels;
    ps.width = width;
    ps.long_rows = L;
    ps.min_len = thr;
    ps.num_chunks = nchunks;
    ps.long_nnz = nl;
}

// ---------------------------------------------------------------------------
// Hot part of Aᵀy: the longest rows of A, per column panel
// ---------------------------------------------------------------------------
namespace {

__global__ void row_len_kernel(const int* __restrict__ rp, int rows, int* __restrict__ len) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x)
        len[i] = rp[i + 1] - rp[i];
}

// Rows of at least `thr` entries are hot (flag 1, plus a trailing 0 for the
// scan); `rest_len` is a row's length in the remaining operand (0 when hot).
__global__ void hot_rows_kernel(const int* __restrict__ rp, int rows, int thr, int* __restrict__ hot,
                                int* __restrict__ rest_len) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= rows; i += gridDim.x * blockDim.x) {
        const int len = i < rows ? rp[i + 1] - rp[i] : 0;
        const bool h = i < rows && len >= thr;
        hot[i] = h ? 1 : 0;
        rest_len[i] = h ? 0 : len;
    }
}

// Per column j of A (row of Aᵀ): entries from hot rows and from the others,
// padded with zeros to `padded` columns (+1 for the scans).
__global__ void split_counts_kernel(const int* __restrict__ trp, const int* __restrict__ trow, int cols,
                                    int padded, const int* __restrict__ hot, int* __restrict__ nh,
                                    int* __restrict__ nr) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j <= padded; j += gridDim.x * blockDim.x) {
        int h = 0, r = 0;
        if (j < cols) {
            for (int k = trp[j]; k < trp[j + 1]; ++k) {
                if (hot[trow[k]]) ++h; else ++r;
            }
        }
        nh[j] = h;
        nr[j] = r;
    }
}

// Copies Aᵀ's entries of hot rows (index among the hot rows, value) and of
// the other rows (the remaining operand), keeping Aᵀ's order.
__global__ void split_copy_kernel(const int* __restrict__ trp, const int* __restrict__ trow,
                                  const float* __restrict__ tval, int cols, const int* __restrict__ hot,
                                  const int* __restrict__ hidx, const int* __restrict__ hoff,
                                  const int* __restrict__ roff, unsigned short* __restrict__ hcol,
                                  float* __restrict__ hval, int* __restrict__ rcol, float* __restrict__ rval) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < cols; j += gridDim.x * blockDim.x) {
        int h = hoff[j], r = roff[j];
        for (int k = trp[j]; k < trp[j + 1]; ++k) {
            const int i = trow[k];
            if (hot[i]) {
                hcol[h] = static_cast<unsigned short>(hidx[i]);
                hval[h] = tval[k];
                ++h;
            } else {
                rcol[r] = i;
                rval[r] = tval[k];
                ++r;
            }
        }
    }
}

__global__ void hot_list_kernel(const int* __restrict__ hot, const int* __restrict__ hidx, int rows,
                                int* __restrict__ list) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x)
        if (hot[i]) list[hidx[i]] = i;
}

__global__ void max_kernel(const int* __restrict__ a, long long n, int* __restrict__ out) {
    int m = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = max(m, a[i]);
    atomicMax(out, m);
}

}  // namespace

void build_panel_hot(const CsrDevice& A, const CsrDevice& AT, const PanelSplit& dual, PanelHot& ph, int gather_cache,
                     int dev, cudaStream_t st) {
    ph = PanelHot{};
    if (!dual.active) return;
    const int rows = A.rows, cols = A.cols;
    if (AT.packed || !AT.col.get() || !AT.val.get()) throw std::logic_error("build_panel_hot needs the flat transpose");
    const size_t limit = panel_smem_limit(dev);
    if (limit <= PanelSmem::off_x) return;
    const int vmax = std::min<long long>((limit - PanelSmem::off_x) / 4, 65536);
    const int panels = dual.panels, width = dual.width;
    const long long padded = (long long)panels * width;
    if (padded + 1 > INT_MAX) return;

    // ---- the hot rows: the vmax longest (ties at the cut left out), at least kPanelHotMinLen long ----
    DevBuf<int> len{size_t(rows)}, len_sorted{size_t(rows)};
    row_len_kernel<<<grid_for_n(rows), kThreads, 0, st>>>(A.row_ptr.get(), rows, len.get());
    PB_CUDA_CHECK(cudaGetLastError());
    {
        size_t tb = 0;
        PB_CUDA_CHECK(cub::DeviceRadixSort::SortKeysDescending(nullptr, tb, len.get(), len_sorted.get(), rows, 0, 32, st));
        DevBuf<unsigned char> temp(tb > 0 ? tb : 1);
        PB_CUDA_CHECK(cub::DeviceRadixSort::SortKeysDescending(temp.get(), tb, len.get(), len_sorted.get(), rows, 0,
                                                               32, st));
        PB_CUDA_CHECK(cudaStreamSynchronize(st));
    }
    int thr = kPanelHotMinLen;
    if (rows > vmax) thr = std::max(thr, read_one(len_sorted.get() + vmax, st) + 1);
    len.reset();
    len_sorted.reset();
    DevBuf<int> hot{size_t(rows) + 1}, hidx{size_t(rows) + 1}, rest_len{size_t(rows) + 1}, rest_rp{size_t(rows) + 1};
    hot_rows_kernel<<<grid_for_n(rows + 1LL), kThreads, 0, st>>>(A.row_ptr.get(), rows, thr, hot.get(),
                                                                  rest_len.get());
    PB_CUDA_CHECK(cudaGetLastError());
    exclusive_sum(hot.get(), hidx.get(), rows + 1LL, st);
    exclusive_sum(rest_len.get(), rest_rp.get(), rows + 1LL, st);
    const int V = read_one(hidx.get() + rows, st);
    if (V <= 0 || V > vmax) return;

    // ---- Aᵀ's entries split by row: hot (per column, in Aᵀ order) and the rest ----
    DevBuf<int> nh{size_t(padded) + 1}, nr{size_t(padded) + 1}, hoff{size_t(padded) + 1}, roff{size_t(padded) + 1};
    split_counts_kernel<<<grid_for_n(padded + 1), kThreads, 0, st>>>(AT.row_ptr.get(), AT.col.get(), cols,
                                                                      int(padded), hot.get(), nh.get(), nr.get());
    PB_CUDA_CHECK(cudaGetLastError());
    {
        DevBuf<int> longest(1);
        PB_CUDA_CHECK(cudaMemsetAsync(longest.get(), 0, 4, st));
        max_kernel<<<grid_for_n(padded), kThreads, 0, st>>>(nh.get(), padded, longest.get());
        PB_CUDA_CHECK(cudaGetLastError());
        if (read_one(longest.get(), st) > kPanelEnt) return;   // a column with more hot entries than a chunk
    }
    exclusive_sum(nh.get(), hoff.get(), padded + 1, st);
    exclusive_sum(nr.get(), roff.get(), padded + 1, st);
    const int nhot = read_one(hoff.get() + padded, st);
    const int nrest = read_one(roff.get() + padded, st);
    if (nhot <= 0) return;
    DevBuf<unsigned short> hcol{size_t(nhot)};
    DevBuf<float> hval{size_t(nhot)};
    CsrDevice& R = ph.rest;
    R.allocate(cols, rows, nrest, /*lo=*/false);
    PB_CUDA_CHECK(cudaMemcpyAsync(R.row_ptr.get(), roff.get(), (size_t(cols) + 1) * 4, cudaMemcpyDeviceToDevice, st));
    split_copy_kernel<<<grid_for_n(cols), kThreads, 0, st>>>(AT.row_ptr.get(), AT.col.get(), AT.val.get(), cols,
                                                            hot.get(), hidx.get(), hoff.get(), roff.get(), hcol.get(),
                                                            hval.get(), R.col.get(), R.val.get());
    PB_CUDA_CHECK(cudaGetLastError());

    // ---- chunks of every panel's columns (segments: the panel's W columns) ----
    DevBuf<int> nch{size_t(panels) + 1};
    PB_CUDA_CHECK(cudaMemsetAsync(nch.get(), 0, nch.bytes(), st));
    chunk_kernel<<<(panels + 63) / 64, 64, 0, st>>>(nh.get(), hoff.get(), width, panels, nch.get(), nullptr,
                                                    nullptr);
    PB_CUDA_CHECK(cudaGetLastError());
    ph.chunk_ptr.alloc(size_t(panels) + 1);
    exclusive_sum(nch.get(), ph.chunk_ptr.get(), panels + 1LL, st);
    const int nchunks = read_one(ph.chunk_ptr.get() + panels, st);
    DevBuf<int4> desc{size_t(nchunks > 0 ? nchunks : 1)};
    chunk_kernel<<<(panels + 63) / 64, 64, 0, st>>>(nh.get(), hoff.get(), width, panels, nullptr,
                                                    ph.chunk_ptr.get(), desc.get());
    PB_CUDA_CHECK(cudaGetLastError());
    ph.rec.alloc(size_t(nchunks) * PanelRec::bytes);
    PB_CUDA_CHECK(cudaMemsetAsync(ph.rec.get(), 0, ph.rec.bytes(), st));
    fill_kernel<<<std::min(nchunks, 65535 * 8), 256, 0, st>>>(desc.get(), nchunks, nh.get(), hoff.get(), width,
                                                             nullptr, hcol.get(), hval.get(), ph.rec.get());
    PB_CUDA_CHECK(cudaGetLastError());
    {
        DevBuf<int> bad(1);
        PB_CUDA_CHECK(cudaMemsetAsync(bad.get(), 0, 4, st));
        check_records_kernel<<<std::min(nchunks, 65535 * 8), 256, 0, st>>>(ph.rec.get(), desc.get(), nchunks,
                                                                          width, width, cols, V, bad.get());
        PB_CUDA_CHECK(cudaGetLastError());
        if (read_one(bad.get(), st)) throw std::logic_error("build_panel_hot: a panel record failed its check");
    }
    ph.hot_row.alloc(size_t(V));
    hot_list_kernel<<<grid_for_n(rows), kThreads, 0, st>>>(hot.get(), hidx.get(), rows, ph.hot_row.get());
    PB_CUDA_CHECK(cudaGetLastError());
    ph.part.alloc(size_t(padded));
    PB_CUDA_CHECK(cudaMemsetAsync(ph.part.get(), 0, ph.part.bytes(), st));

    // ---- the remaining operand: hot gather slots among the other rows, then tile records ----
    R.finalize(st);
    if (gather_cache >= 0) R.select_hot(rest_rp.get(), rows, dev, st);
    R.pack(st);
    PB_CUDA_CHECK(cudaStreamSynchronize(st));   // temporaries are freed on return

    ph.active = true;
    ph.panels = panels;
    ph.width = width;
    ph.hot_rows = V;
    ph.min_len = thr;
    ph.num_chunks = nchunks;
    ph.hot_nnz = nhot;
}

}  // namespace pb
