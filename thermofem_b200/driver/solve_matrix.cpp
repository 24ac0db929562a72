// solve-matrix -- manufactured-solution check of the solve path on a Matrix
// Market file, through the C ABI (example/solve-matrix.cu:54-180 of the
// reference: same arguments, same key=value report, same exit codes).
//
//   solve-matrix path [amg|identity] [v|w|f]
//
// The known solution x_i = 1 + 0.25 sin(0.013 i) + 0.125 cos(0.007 i) gives
// b = A x on the host (long double sums); right-preconditioned BiCGStab in
// FP64 (rtol 1e-8, atol 0, 1000 iterations, refresh every 50) solves from a
// zero guess, and the host checks the true relative residual (<= 1.01e-8)
// and the relative solution error (<= 1e-4).  Exit 0 when both pass, 2 on a
// numeric failure, 1 on an input or execution error (message on stderr as
// error=...).  THERMOFEM_B200_HIERARCHY=f32 runs the AMG cycle in FP32 under
// the FP64 outer loop (the default is the reference's FP64 hierarchy).
// THERMOFEM_B200_DRIVER_EXTRA=1 appends, after the reference's keys,
// precision=, device_solve_ms= (CUDA events around the solve),
// operator_spmv_gbs= (algorithmic bytes of the FP64 operator SpMV over the
// mean of 20 event-timed launches), operator_spmv_roofline_fraction= and
// peak_gbs= (THERMOFEM_B200_HBM_GBS, else 6650 GB/s), peak_source=.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "thermofem_b200.h"

namespace {

void ok(int status) {
    if (status == TF_OK) return;
    const char *m = tf_last_error();
    const std::string msg = m && *m ? m : tf_status_string(status);
    if (status == TF_ERR_INVALID) throw std::invalid_argument(msg);
    if (status == TF_ERR_LENGTH) throw std::length_error(msg);
    if (status == TF_ERR_LOGIC) throw std::logic_error(msg);
    throw std::runtime_error(msg);
}

void cuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

const char *status_name(int s) {
    switch (s) {
        case TF_CONVERGED: return "Converged";
        case TF_MAX_ITERATIONS: return "MaxIterations";
        case TF_BREAKDOWN: return "Breakdown";
        case TF_NONFINITE: return "NonFinite";
        default: return "Unknown";
    }
}

// y = A x on the host with long double sums (the independent check).
std::vector<double> host_multiply(const tf_host_csr &a, const std::vector<double> &x) {
    std::vector<double> y(static_cast<size_t>(a.rows));
    for (int r = 0; r < a.rows; ++r) {
        long double s = 0;
        for (int32_t j = a.offsets[r]; j < a.offsets[r + 1]; ++j)
            s += static_cast<long double>(a.values[j]) * x[static_cast<size_t>(a.indices[j])];
        y[static_cast<size_t>(r)] = static_cast<double>(s);
    }
    return y;
}

// Device copy of one host array.
template <class T>
struct Device {
    T *p{nullptr};
    explicit Device(const T *src, size_t n) {
        cuda(cudaMalloc(&p, (n ? n : 1) * sizeof(T)), "cudaMalloc");
        if (n && src) cuda(cudaMemcpy(p, src, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy");
    }
    ~Device() { cudaFree(p); }
    Device(const Device &) = delete;
    Device &operator=(const Device &) = delete;
};

// The performance keys appended on request: precision, device solve time and
// the operator SpMV's achieved bandwidth against the HBM peak.
void report_extra(tf_ctx *ctx, tf_solver *solver, size_t n, size_t nnz, bool mixed) {
    int sliced = 0;
    int64_t entries = 0;
    ok(tf_solver_spmv_layout(solver, &sliced, &entries));
    // sliced copy: values + 2-byte offsets per entry, one start per 32-row
    // slice, x and y once; CSR: values + 2-byte columns, row offsets, x, y
    const double bytes = sliced ? double(entries) * 10 + double((n + 31) / 32 + 1) * 4 + double(n) * 16
                                : double(nnz) * 10 + double(n) * 20 + 4;
    Device<double> x(nullptr, n), y(nullptr, n);
    cuda(cudaMemset(x.p, 0, n * sizeof(double)), "cudaMemset");
    auto stream = static_cast<cudaStream_t>(tf_ctx_stream(ctx));
    for (int k = 0; k < 3; ++k) ok(tf_solver_spmv(solver, x.p, y.p));
    cudaEvent_t e0, e1;
    cuda(cudaEventCreate(&e0), "cudaEventCreate");
    cuda(cudaEventCreate(&e1), "cudaEventCreate");
    constexpr int kReps = 20;
    cuda(cudaEventRecord(e0, stream), "cudaEventRecord");
    for (int k = 0; k < kReps; ++k) ok(tf_solver_spmv(solver, x.p, y.p));
    cuda(cudaEventRecord(e1, stream), "cudaEventRecord");
    cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
    float ms = 0;
    cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double gbs = bytes / (double(ms) / kReps * 1e-3) / 1e9;
    const char *peak_env = std::getenv("THERMOFEM_B200_HBM_GBS");
    const double peak = peak_env ? std::atof(peak_env) : 6650.0;
    std::cout << "precision=" << (mixed ? "f32_hierarchy_f64_outer" : "f64")
              << "\ndevice_solve_ms=" << tf_solver_last_apply_ms(solver) << "\noperator_spmv_layout="
              << (sliced ? "sliced" : "csr") << "\noperator_spmv_gbs=" << gbs
              << "\noperator_spmv_roofline_fraction=" << (peak > 0 ? gbs / peak : 0.0) << "\npeak_gbs=" << peak
              << "\npeak_source=" << (peak_env ? "THERMOFEM_B200_HBM_GBS" : "fallback") << '\n';
}

}  // namespace

int main(int argc, char **argv) {
    using Clock = std::chrono::steady_clock;
    std::cout << std::unitbuf << std::setprecision(12);
    tf_host_csr host{};
    tf_ctx *ctx = nullptr;
    tf_solver *solver = nullptr;
    int code = 1;
    try {
        if (argc < 2 || argc > 4) throw std::invalid_argument("Usage: solve-matrix path [amg|identity] [v|w|f]");
        const std::string mode = argc >= 3 ? argv[2] : "amg";
        const std::string cycle = argc == 4 ? argv[3] : "v";
        if (cycle != "v" && cycle != "w" && cycle != "f") throw std::invalid_argument("Unknown cycle");
        if (mode != "amg" && mode != "identity") throw std::invalid_argument("Unknown preconditioner");
        const auto begin = Clock::now();
        {
            std::ifstream probe(argv[1]);
            if (!probe) throw std::runtime_error("Cannot open matrix file");
        }
        ok(tf_read_matrix_market_file(argv[1], &host));
        if (host.rows <= 0 || host.rows != host.cols) throw std::invalid_argument("Expected nonempty square matrix");
        const auto loaded = Clock::now();
        const size_t n = static_cast<size_t>(host.rows);
        std::cout << "matrix=" << argv[1] << "\nrows=" << n << "\nnnz=" << host.nnz << "\npreconditioner=" << mode
                  << "\nread_seconds=" << std::chrono::duration<double>(loaded - begin).count() << '\n';
        std::vector<double> exact(n), x(n, 0.0);
        for (size_t i = 0; i < n; ++i)
            exact[i] = 1.0 + 0.25 * std::sin(double(i) * 0.013) + 0.125 * std::cos(double(i) * 0.007);
        const std::vector<double> b = host_multiply(host, exact);
        int device = 0;
        cuda(cudaGetDevice(&device), "cudaGetDevice");
        cudaDeviceProp prop{};
        cuda(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
        int runtime = 0;
        cuda(cudaRuntimeGetVersion(&runtime), "cudaRuntimeGetVersion");
        std::cout << "device=" << device << "\ngpu=" << prop.name << "\ncuda_runtime=" << runtime
                  << "\nrtol=" << 1e-8 << "\natol=0\nmax_iterations=1000\nrefresh_interval=50\n";

        ok(tf_ctx_create(device, nullptr, &ctx));
        const size_t nnz = static_cast<size_t>(host.nnz);
        Device<int32_t> d_off(host.offsets, n + 1), d_idx(host.indices, nnz);
        Device<double> d_val(host.values, nnz), d_b(b.data(), n), d_x(x.data(), n);
        tf_csr a{static_cast<int64_t>(n), static_cast<int64_t>(n), static_cast<int64_t>(nnz), TF_I32, TF_F64,
                 d_off.p, d_idx.p, d_val.p};
        tf_amg_options amg;
        tf_amg_options_default(&amg);
        amg.cycle = cycle == "v" ? TF_CYCLE_V : (cycle == "w" ? TF_CYCLE_W : TF_CYCLE_F);
        const char *h = std::getenv("THERMOFEM_B200_HIERARCHY");
        if (h && std::string(h) == "f32") amg.hierarchy_type = TF_F32;
        tf_solver_options opt;
        tf_solver_options_default(TF_F64, &opt);
        opt.relative_tolerance = 1e-8;
        ok(tf_solver_create(ctx, TF_SOLVER_BICGSTAB, TF_F64, TF_I32, &opt,
                            mode == "amg" ? TF_PRECOND_AMG : TF_PRECOND_IDENTITY, &amg, &solver));
        std::cout << "phase=setup\n";
        const auto setup_begin = Clock::now();
        ok(tf_solver_setup(solver, &a));
        const auto setup_end = Clock::now();
        std::cout << "setup_seconds=" << std::chrono::duration<double>(setup_end - setup_begin).count() << '\n';
        if (mode == "amg") {
            tf_amg *m = tf_solver_amg(solver);
            const int levels = tf_amg_level_count(m);
            std::cout << "cycle=" << cycle << "\nlevels=" << levels << "\nstop_reason=" << tf_amg_stop_reason(m)
                      << "\ncoarse_solver=" << tf_amg_coarse_solver(m) << '\n';
            size_t total_rows = 0, total_nnz = 0;
            for (int d = 0; d < levels; ++d) {
                int64_t rows = 0, lnnz = 0;
                int32_t hist[4];
                ok(tf_amg_level_stats(m, d, &rows, &lnnz, hist));
                total_rows += static_cast<size_t>(rows);
                total_nnz += static_cast<size_t>(lnnz);
                std::cout << "level=" << d << " rows=" << rows << " nnz=" << lnnz << " aggregates=";
                for (int k = 0; k < 4; ++k) std::cout << hist[k] << ',';
                std::cout << '\n';
            }
            std::cout << "grid_complexity=" << double(total_rows) / n
                      << "\noperator_complexity=" << double(total_nnz) / nnz << '\n';
        }
        std::cout << "phase=solve\n";
        tf_solve_result report{};
        ok(tf_solver_apply(solver, d_b.p, d_x.p, 0, &report));
        const auto solved = Clock::now();
        cuda(cudaMemcpy(x.data(), d_x.p, n * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
        const std::vector<double> product = host_multiply(host, x);
        long double rr = 0, bb = 0, ee = 0, xx = 0;
        bool finite = true;
        for (size_t i = 0; i < n; ++i) {
            finite = finite && std::isfinite(x[i]) && std::isfinite(product[i]);
            const long double r = static_cast<long double>(b[i]) - product[i];
            const long double e = static_cast<long double>(x[i]) - exact[i];
            rr += r * r;
            bb += static_cast<long double>(b[i]) * b[i];
            ee += e * e;
            xx += static_cast<long double>(exact[i]) * exact[i];
        }
        const auto host_residual = std::sqrt(rr / (bb > 0 ? bb : 1));
        const auto solution_error = std::sqrt(ee / xx);
        std::cout << "status=" << status_name(report.status) << "\niterations=" << report.iterations
                  << "\nsolve_seconds=" << std::chrono::duration<double>(solved - setup_end).count()
                  << "\nreported_relative_residual=" << report.relative_residual
                  << "\nhost_relative_residual=" << host_residual << "\nrelative_solution_error=" << solution_error
                  << '\n';
        const bool passed =
            finite && report.status == TF_CONVERGED && host_residual <= 1.01e-8 && solution_error <= 1e-4;
        std::cout << "validation=" << (passed ? "PASS" : "FAIL") << '\n';
        const char *extra = std::getenv("THERMOFEM_B200_DRIVER_EXTRA");
        if (extra && extra[0] == '1') report_extra(ctx, solver, n, nnz, mode == "amg" && h && std::string(h) == "f32");
        code = passed ? 0 : 2;
    } catch (const std::exception &e) {
        std::cerr << "error=" << e.what() << '\n';
        code = 1;
    }
    if (solver) tf_solver_destroy(solver);
    if (ctx) tf_ctx_destroy(ctx);
    if (host.offsets) tf_host_csr_free(&host);
    return code;
}
