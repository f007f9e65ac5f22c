// certificate.cuh — FP64 certificates of points of many LPs (certificate.cu).
#pragma once

#include <vector>

#include "csr_device.cuh"
#include "epilogues.cuh"

namespace pb {

class CertificateBatch {
public:
    // Packs the LPs once (FP64 values split into FP32 hi + lo, transpose built
    // on the device).
    CertificateBatch(const pramaan_lp* lps, int count, int device);
    ~CertificateBatch();
    CertificateBatch(const CertificateBatch&) = delete;
    CertificateBatch& operator=(const CertificateBatch&) = delete;

    // out[k] = certificate of points[k] for LP k (x NULL: the cold start
    // clamp(0, l, u); y NULL: 0).
    void evaluate(const pramaan_warm_start* points, pramaan_certificate* out);

private:
    int dev_ = 0, count_ = 0, m_ = 0, n_ = 0, nnz_ = 0;
    int rchunks_ = 0, cchunks_ = 0;
    cudaStream_t st_ = nullptr;
    std::vector<int> r0_, c0_;
    std::vector<double> offset_;
    CsrDevice A_, AT_;
    DevBuf<double> rlo_, rhi_, vlo_, vhi_, cmin_, cmod_;
    DevBuf<int> rbegin_, rfirst_, cbegin_, cfirst_, status_;
    DevBuf<double> x_, y_, act_, aty_, contrib_, chunk_out_, lp_out_;
};

}  // namespace pb
