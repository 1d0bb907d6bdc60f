// spd.cuh — sparse SPD factorisation on the GPU behind the reference's ISpdSolver seam
// (Solver/Linear/ISpdSolver.cs:24-41; replaces CudssSolver.cs:105-145).
//
// The reference's GPU backend is NVIDIA cuDSS 0.8.0, which this toolchain does not ship. The factorisation
// stays a vendor library call: cuSOLVER's sparse Cholesky (csrchol: symbolic analysis once per pattern, numeric
// factorisation and triangular solves on the device), after a nested-dissection order (METIS, cuSOLVER's host
// helper) on the 3x3 node graph. Values never leave the device: the full-CSC values the assembly produced are
// gathered into the permuted CSR the factorisation reads by one kernel.
#pragma once
#include <cusolverSp.h>
#include <cusolverSp_LOWLEVEL_PREVIEW.h>
#include <cusparse.h>

#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "runtime.cuh"

namespace ifea {

inline void cusolver_check(cusolverStatus_t s, const char *what)
{
    if (s != CUSOLVER_STATUS_SUCCESS)
        throw Failure(IFEA_DIVERGED, std::string(what) + " failed (cuSOLVER status " + std::to_string((int)s) + ")");
}
inline void cusparse_check(cusparseStatus_t s, const char *what)
{
    if (s != CUSPARSE_STATUS_SUCCESS)
        throw Failure(IFEA_CUDA_ERROR, std::string(what) + " failed (cuSPARSE status " + std::to_string((int)s) + ")");
}

static __global__ void k_gather(int n, const int32_t *__restrict__ src, const double *__restrict__ in, double *__restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = in[src[i]];
}
static __global__ void k_scatter(int n, const int32_t *__restrict__ dst, const double *__restrict__ in, double *__restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[dst[i]] = in[i];
}
static __global__ void k_finite_check(int n, const double *x, int *flag)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (!isfinite(x[i])) atomicExch(flag, 1);
}

class GpuSpd {
public:
    explicit GpuSpd(cudaStream_t s) : stream_(s)
    {
        cusolver_check(cusolverSpCreate(&h_), "cusolverSpCreate");
        cusolver_check(cusolverSpSetStream(h_, s), "cusolverSpSetStream");
        cusparse_check(cusparseCreateMatDescr(&descr_), "cusparseCreateMatDescr");
        cusparseSetMatType(descr_, CUSPARSE_MATRIX_TYPE_GENERAL);
        cusparseSetMatIndexBase(descr_, CUSPARSE_INDEX_BASE_ZERO);
        flag_.resize(1);
    }
    ~GpuSpd()
    {
        if (info_) cusolverSpDestroyCsrcholInfo(info_);
        if (descr_) cusparseDestroyMatDescr(descr_);
        if (h_) cusolverSpDestroy(h_);
    }
    GpuSpd(const GpuSpd &) = delete;
    GpuSpd &operator=(const GpuSpd &) = delete;

    void set_stream(cudaStream_t s)
    {
        stream_ = s;
        cusolver_check(cusolverSpSetStream(h_, s), "cusolverSpSetStream");
    }
    int n() const { return n_; }
    bool analyzed() const { return analyzed_; }
    bool factored() const { return factored_; }
    int64_t factor_nonzeros() const { return factor_nnz_; }

    // Symbolic analysis of a full symmetric CSC pattern (host arrays). block = 3 orders the 3x3 node graph.
    void analyze(int n, const int32_t *col_ptr, const int32_t *row_idx, int block)
    {
        if (n <= 0) throw Failure(IFEA_INPUT_INVALID, "empty system");
        n_ = n;
        factored_ = false;
        analyzed_ = false;
        if (block < 1 || n % block) block = 1;
        int nb = n / block;
        // graph of the blocks (no self loops) for the nested-dissection order
        std::vector<int> gp(nb + 1, 0), gi;
        std::vector<int> mark(nb, -1);
        for (int b = 0; b < nb; b++) {
            int d = b * block;
            for (int32_t p = col_ptr[d]; p < col_ptr[d + 1]; p++) {
                int o = row_idx[p] / block;
                if (o == b || mark[o] == b) continue;
                mark[o] = b;
                gi.push_back(o);
            }
            gp[b + 1] = (int)gi.size();
        }
        std::vector<int> pnode(nb);
        if (gi.empty()) {
            std::iota(pnode.begin(), pnode.end(), 0);
        } else {
            cusolver_check(cusolverSpXcsrmetisndHost(h_, nb, (int)gi.size(), descr_, gp.data(), gi.data(), nullptr, pnode.data()),
                           "cusolverSpXcsrmetisndHost");
        }
        perm_h_.resize(n);
        std::vector<int> pinv(n);
        for (int k = 0; k < nb; k++)
            for (int c = 0; c < block; c++) perm_h_[k * block + c] = pnode[k] * block + c;
        for (int k = 0; k < n; k++) pinv[perm_h_[k]] = k;
        // permuted CSR: row r = old column perm[r], entries sorted by new column index
        std::vector<int> rp(n + 1, 0), ci, src;
        int64_t nnz = col_ptr[n];
        ci.reserve(nnz);
        src.reserve(nnz);
        std::vector<std::pair<int, int>> row;
        for (int r = 0; r < n; r++) {
            int d = perm_h_[r];
            row.clear();
            for (int32_t p = col_ptr[d]; p < col_ptr[d + 1]; p++) row.emplace_back(pinv[row_idx[p]], (int)p);
            std::sort(row.begin(), row.end());
            for (auto &e : row) { ci.push_back(e.first); src.push_back(e.second); }
            rp[r + 1] = (int)ci.size();
        }
        nnz_ = (int)ci.size();
        d_rp_.upload(rp.data(), rp.size(), stream_);
        d_ci_.upload(ci.data(), ci.size(), stream_);
        d_src_.upload(src.data(), src.size(), stream_);
        d_perm_.upload(perm_h_.data(), perm_h_.size(), stream_);
        d_vals_.resize(nnz_);
        d_pb_.resize(n);
        d_px_.resize(n);
        if (info_) cusolverSpDestroyCsrcholInfo(info_);
        info_ = nullptr;
        cusolver_check(cusolverSpCreateCsrcholInfo(&info_), "cusolverSpCreateCsrcholInfo");
        cusolver_check(cusolverSpXcsrcholAnalysis(h_, n_, nnz_, descr_, d_rp_, d_ci_, info_), "cusolverSpXcsrcholAnalysis");
        d_vals_.zero(stream_);
        size_t internal = 0, work = 0;
        cusolver_check(cusolverSpDcsrcholBufferInfo(h_, n_, nnz_, descr_, d_vals_, d_rp_, d_ci_, info_, &internal, &work),
                       "cusolverSpDcsrcholBufferInfo");
        d_work_.resize(std::max<size_t>(work, 16));
        factor_nnz_ = (int64_t)(internal / sizeof(double));
        analyzed_ = true;
    }

    // Numeric factorisation of device values given in the order of the analysed full CSC pattern.
    void factorize(const double *d_full_vals)
    {
        if (!analyzed_) throw Failure(IFEA_BAD_STATE, "Analyze must be called first.");
        factored_ = false;
        k_gather<<<grid(nnz_), 256, 0, stream_>>>(nnz_, d_src_, d_full_vals, d_vals_);
        cusolver_check(cusolverSpDcsrcholFactor(h_, n_, nnz_, descr_, d_vals_, d_rp_, d_ci_, info_, d_work_),
                       "cusolverSpDcsrcholFactor");
        int pos = -1;
        cusolver_check(cusolverSpDcsrcholZeroPivot(h_, info_, 0.0, &pos), "cusolverSpDcsrcholZeroPivot");
        if (pos >= 0) {
            int row = perm_h_[pos];
            throw Failure(IFEA_NOT_SPD, "Stiffness matrix not positive definite at equation " + std::to_string(row) +
                                            ". The billet is probably unrestrained.");
        }
        factored_ = true;
    }

    // x = A^-1 b on the device (b and x may alias).
    void solve(const double *d_b, double *d_x)
    {
        if (!factored_) throw Failure(IFEA_BAD_STATE, "Factorize must be called first.");
        k_gather<<<grid(n_), 256, 0, stream_>>>(n_, d_perm_, d_b, d_pb_);
        cusolver_check(cusolverSpDcsrcholSolve(h_, n_, d_pb_, d_px_, info_, d_work_), "cusolverSpDcsrcholSolve");
        k_scatter<<<grid(n_), 256, 0, stream_>>>(n_, d_perm_, d_px_, d_x);
    }

    // Non-finite entries in x -> MatrixNotPositiveDefiniteException(-1) (CudssSolver.cs:141-144).
    void check_finite(const double *d_x)
    {
        flag_.zero(stream_);
        k_finite_check<<<grid(n_), 256, 0, stream_>>>(n_, d_x, flag_);
        int f = 0;
        flag_.download(&f, 1, stream_);
        cuda_check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
        if (f) throw Failure(IFEA_NOT_SPD, "Stiffness matrix not positive definite at equation -1 (pivot NaN).");
    }

private:
    static int grid(int n) { return std::max(1, std::min((n + 255) / 256, 4 * 148)); }
    cudaStream_t stream_;
    cusolverSpHandle_t h_ = nullptr;
    cusparseMatDescr_t descr_ = nullptr;
    csrcholInfo_t info_ = nullptr;
    int n_ = 0, nnz_ = 0;
    bool analyzed_ = false, factored_ = false;
    int64_t factor_nnz_ = 0;
    std::vector<int> perm_h_;
    DBuf<int> d_rp_, d_ci_, d_src_, d_perm_, flag_;
    DBuf<double> d_vals_, d_pb_, d_px_;
    DBuf<char> d_work_;
};

}  // namespace ifea
