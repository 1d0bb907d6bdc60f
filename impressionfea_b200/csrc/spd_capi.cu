// spd_capi.cu — C ABI of the GPU sparse SPD solver (ifea_spd_*), shaped like the reference's ISpdSolver
// (Solver/Linear/ISpdSolver.cs:24-41) so a CudssSolver-style P/Invoke backend can bind it directly.
#include <string>
#include <vector>

#include "multifrontal.cuh"

struct ifea_spd {
    cudaStream_t st = nullptr;
    ifea::MfSolver *s = nullptr;
    ifea::DBuf<double> vals, b, x;
    std::vector<int32_t> col_ptr;
    int n = 0;
    int64_t nnz = 0;
    std::string err, name;
};

template <typename F>
static ifea_status spd_guard(ifea_spd *h, F &&f)
{
    if (!h) return IFEA_INPUT_INVALID;
    try {
        f(*h);
        h->err.clear();
        return IFEA_OK;
    } catch (ifea::Failure &e) {
        h->err = e.what();
        return e.status;
    } catch (std::exception &e) {
        h->err = e.what();
        return IFEA_CUDA_ERROR;
    }
}

extern "C" {

ifea_status ifea_spd_create(ifea_spd **out)
{
    if (!out) return IFEA_INPUT_INVALID;
    *out = nullptr;
    ifea_spd *h = new ifea_spd;
    try {
        ifea::cuda_check(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking), "cudaStreamCreate");
        h->s = new ifea::MfSolver(h->st);
        cudaDeviceProp prop;
        ifea::cuda_check(cudaGetDeviceProperties(&prop, 0), "cudaGetDeviceProperties");
        h->name = std::string("multifrontal sparse Cholesky (GPU · ") + prop.name + ")";
    } catch (ifea::Failure &e) {
        delete h->s;
        if (h->st) cudaStreamDestroy(h->st);
        delete h;
        return e.status;
    }
    *out = h;
    return IFEA_OK;
}

void ifea_spd_destroy(ifea_spd *h)
{
    if (!h) return;
    delete h->s;
    h->vals.release();
    h->b.release();
    h->x.release();
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

const char *ifea_spd_last_error(const ifea_spd *h) { return h ? h->err.c_str() : "null handle"; }
const char *ifea_spd_name(const ifea_spd *h) { return h ? h->name.c_str() : ""; }

// ISpdSolver.Analyze(n, colPtr, rowIdx): symbolic analysis of a full symmetric CSC pattern.
ifea_status ifea_spd_analyze(ifea_spd *h, int32_t n, const int32_t *col_ptr, const int32_t *row_idx)
{
    if (!col_ptr || !row_idx || n <= 0) return IFEA_INPUT_INVALID;
    return spd_guard(h, [&](ifea_spd &s) {
        s.n = n;
        s.nnz = col_ptr[n];
        s.col_ptr.assign(col_ptr, col_ptr + n + 1);
        s.s->analyze(n, col_ptr, row_idx, 1);
        s.vals.resize(s.nnz);
        s.b.resize(n);
        s.x.resize(n);
    });
}

// ISpdSolver.Factorize(values): values in the order of the analysed full CSC pattern (host).
ifea_status ifea_spd_factorize(ifea_spd *h, const double *values)
{
    if (!values) return IFEA_INPUT_INVALID;
    return spd_guard(h, [&](ifea_spd &s) {
        if (!s.s->analyzed()) throw ifea::Failure(IFEA_BAD_STATE, "Analyze must be called first.");
        s.vals.upload(values, s.nnz, s.st);
        s.s->factorize(s.vals);
    });
}

// ISpdSolver.Solve(b, x) (host).
ifea_status ifea_spd_solve(ifea_spd *h, const double *b, double *x)
{
    if (!b || !x) return IFEA_INPUT_INVALID;
    return spd_guard(h, [&](ifea_spd &s) {
        s.b.upload(b, s.n, s.st);
        s.s->solve(s.b, s.x);
        s.s->check_finite(s.x);
        s.x.download(x, s.n, s.st);
        ifea::cuda_check(cudaStreamSynchronize(s.st), "cudaStreamSynchronize");
    });
}

int64_t ifea_spd_factor_nonzeros(const ifea_spd *h) { return h && h->s ? h->s->factor_nonzeros() : 0; }

const char *ifea_version(void) { return "ifea-b200 0.1 (sm_100a, FP64 path)"; }

}  // extern "C"
