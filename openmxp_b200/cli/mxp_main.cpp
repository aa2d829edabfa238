// mxp: command-line driver of the single-GPU solve, with the reference's
// output (main.cpp:281-297 banner, 600-657 run lines, 670-705 summary and
// "Submission Output" block; iterative_refinement.hpp:158-161 IR lines;
// timer.hpp:58-85,185-208 timer table), so tooling that reads the reference's
// output reads this program's too.
//
//   mxp N B [P Q] [-form fp16|bf16x2|fp8] [-ir classic|gmres] [-alt 0|1|2]
//       [-seed S] [-diag 0|1] [-maxit M] [-warmup W] [-sys NAME] [--job-id ID]
//
// P x Q must be 1 x 1 (one GPU).  -alt 0 solves the panels with the SIMT TRSM
// (the reference's "Default Trsm"), 1 and 2 with the tensor-core TRSM by
// inverse (its "Alt-Trsm" family): 1 as three split-BF16 products (near FP32),
// 2 as one BF16 product (the low-precision GEMM of the reference's alt 2).
// Options the single-GPU path does not have are reported as ignored, as the
// reference does with unknown options.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>

#include "mxp.h"

namespace {

struct Args {
    int n = 8192, b = 256, p = 1, q = 1;
    int form = MXP_FORM_FP16;
    int ir = MXP_IR_CLASSIC;
    int alt = 1;
    uint64_t seed = 42;  // main.cpp:325
    int diag = MXP_DIAG_ROWSUM;
    int maxit = 50;
    int warmup = 0;
    int jobid = 0;
    std::string sys = "B200";
};

bool is_int(const char *s) {
    if (!s || !*s) return false;
    for (const char *c = s; *c; ++c)
        if (*c < '0' || *c > '9') return false;
    return true;
}

void parse(int argc, char **argv, Args &a) {
    int i = 1;
    int *pos[4] = {&a.n, &a.b, &a.p, &a.q};
    for (int k = 0; k < 4 && i < argc && is_int(argv[i]); ++k, ++i) *pos[k] = std::atoi(argv[i]);
    for (; i < argc; ++i) {
        const char *o = argv[i];
        const bool has = i + 1 < argc;
        if (!std::strcmp(o, "-form") && has) {
            const char *v = argv[++i];
            a.form = !std::strcmp(v, "fp8") ? MXP_FORM_FP8 : !std::strcmp(v, "bf16x2") ? MXP_FORM_BF16X2 : MXP_FORM_FP16;
        } else if (!std::strcmp(o, "-ir") && has) {
            a.ir = !std::strcmp(argv[++i], "gmres") ? MXP_IR_GMRES : MXP_IR_CLASSIC;
        } else if (!std::strcmp(o, "-alt") && has) {
            a.alt = std::atoi(argv[++i]);
        } else if (!std::strcmp(o, "-seed") && has) {
            a.seed = std::strtoull(argv[++i], nullptr, 10);
        } else if (!std::strcmp(o, "-diag") && has) {
            a.diag = std::atoi(argv[++i]) ? MXP_DIAG_055_PLUS1 : MXP_DIAG_ROWSUM;
        } else if (!std::strcmp(o, "-maxit") && has) {
            a.maxit = std::atoi(argv[++i]);
        } else if (!std::strcmp(o, "-warmup") && has) {
            a.warmup = std::atoi(argv[++i]);
        } else if (!std::strcmp(o, "-sys") && has) {
            a.sys = argv[++i];
        } else if (!std::strcmp(o, "--job-id") && has) {
            a.jobid = std::atoi(argv[++i]);
        } else if (!std::strcmp(o, "--help") || !std::strcmp(o, "-h")) {
            std::printf("usage: mxp N B [P Q] [-form fp16|bf16x2|fp8] [-ir classic|gmres] [-alt 0|1|2]\n"
                        "           [-seed S] [-diag 0|1] [-maxit M] [-warmup W] [-sys NAME] [--job-id ID]\n");
            std::exit(0);
        } else {
            std::printf("Ignoring unknown option: %s\n", o);
        }
    }
}

std::string now() {
    std::time_t t = std::time(nullptr);
    std::string s = std::ctime(&t);
    if (!s.empty() && s.back() == '\n') s.pop_back();
    return s;
}

int die(const char *what, mxp_status s) {
    std::fprintf(stderr, "mxp: %s failed: %s (status %d)\n", what, mxp_last_error_string(), (int)s);
    return 2;
}

}  // namespace

int main(int argc, char **argv) {
    Args a;
    parse(argc, argv, a);
    std::printf("===============================================================================\n");
    std::printf("OpenMxP - High Performance Mixed Precision Benchmark - NCCS/OLCF\n");
    std::printf("===============================================================================\n");
    std::printf("Build Info: %s\n", mxp_version());
    std::printf("Running configuration:\n");
    std::printf("\tRanks = 1\n");
    if (std::getenv("CMD")) std::printf("\t%s\n", std::getenv("CMD"));
    if (std::getenv("NOTE")) std::printf("\tNOTE: %s\n", std::getenv("NOTE"));
    if (a.p * a.q != 1) {
        std::printf("\tCan't run this grid configuration\n");
        return 1;
    }
    if (a.n <= 0 || a.b <= 0 || a.n % a.b) {
        std::printf("\tN must be a positive multiple of B\n");
        return 1;
    }
    const char *forms[] = {"FP16", "BF16x2", "FP8"};
    const char *alts[] = {"Default Trsm", "Alt-Trsm", "Alt2"};
    std::printf("\t%s Schur update\n", forms[a.form]);
    std::printf("\t%s Method\n", alts[a.alt < 0 || a.alt > 2 ? 1 : a.alt]);
    std::printf("\t%s refinement\n", a.ir == MXP_IR_GMRES ? "GMRES" : "Classic");

    const int n = a.n, b = a.b;
    float *A = nullptr;
    double *d = nullptr, *rs = nullptr, *rhs = nullptr, *x = nullptr;
    if (cudaMalloc(&A, sizeof(float) * (size_t)n * n) != cudaSuccess ||
        cudaMalloc(&d, sizeof(double) * n) != cudaSuccess || cudaMalloc(&rs, sizeof(double) * n) != cudaSuccess ||
        cudaMalloc(&rhs, sizeof(double) * n) != cudaSuccess || cudaMalloc(&x, sizeof(double) * n) != cudaSuccess) {
        std::fprintf(stderr, "mxp: device allocation of %.1f GB failed\n", 4.0 * n * (double)n / 1e9);
        return 2;
    }
    mxp_workspace *ws = nullptr;
    mxp_status s = mxp_workspace_create(n, b, a.form, 0, &ws);
    if (s != MXP_OK) return die("workspace_create", s);
    mxp_workspace_set_option(ws, MXP_OPT_TRSM_TENSOR, a.alt == 0 ? 0 : 1);
    mxp_workspace_set_option(ws, MXP_OPT_TRSM_SINGLE, a.alt == 2 ? 1 : 0);
    std::printf("\tjobid=%d\n", a.jobid);
    std::printf("\tn=%d ln=%d b=%d r=%d c=%d epoch_size=%d\n", n, n, b, 0, 0, b);

    mxp_lu_stats lu{};
    mxp_ir_stats ir{};
    const double *rowsum = a.diag == MXP_DIAG_ROWSUM ? nullptr : rs;
    for (int w = 0; w <= a.warmup; ++w) {
        s = mxp_matgen(n, a.seed, a.diag, A, n, d, rs, rhs, nullptr);
        if (s != MXP_OK) return die("matgen", s);
        cudaDeviceSynchronize();
        if (w < a.warmup) {
            s = mxp_solve(n, b, a.seed, A, n, d, rowsum, rhs, x, a.maxit, a.ir, ws, nullptr, &lu, &ir);
            if (s != MXP_OK && s != MXP_NOT_CONVERGED) return die("warm-up solve", s);
        }
    }
    const std::string begin = now();
    std::printf("#BEGIN_: %s\n", begin.c_str());
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    cudaEventRecord(e0, nullptr);
    s = mxp_panel_lu(n, b, A, n, ws, nullptr, &lu);
    if (s != MXP_OK) return die("panel_lu", s);
    cudaEventRecord(e1, nullptr);
    std::printf("\nIR Start\n");
    s = mxp_iterative_refinement(n, a.seed, A, n, d, rowsum, rhs, x, 0.0, a.maxit, a.ir, ws, nullptr, &ir);
    cudaEventRecord(e2, nullptr);
    cudaEventSynchronize(e2);
    if (s != MXP_OK && s != MXP_NOT_CONVERGED) return die("iterative_refinement", s);
    for (int it = 0; it <= ir.iterations && it < 64; ++it)
        std::printf("# iterative refinement: step=%d, residual=%e, hpl-harness=%f\n", it, ir.history_residual[it],
                    ir.history[it]);
    float ms_lu = 0.0f, ms_ir = 0.0f;
    cudaEventElapsedTime(&ms_lu, e0, e1);
    cudaEventElapsedTime(&ms_ir, e1, e2);
    std::printf("\t IR Time %.2f sec\n", ms_ir / 1e3);

    const double t = (ms_lu + ms_ir) / 1e3;
    const double flops = 2.0 / 3.0 * (double)n * n * n + 1.5 * (double)n * n;
    const bool conv = s == MXP_OK && ir.converged;
    const double resid = conv ? ir.residual : -1.0, harness = conv ? ir.hpl_harness : -1.0;
    std::printf("#END___: %s\n", now().c_str());
    std::printf("%.3f sec. %.3f GFlop/s resid = %20.15e hpl-harness = %.9f TFlop/s per GPU = %.3f\n", t,
                flops / t * 1e-9, resid, harness, flops / t * 1e-12);
    std::printf("===================================\n");
    std::printf("NCCS/OLCF Mixed Precision Benchmark\n");
    std::printf("Code   : OpenMxP\n");
    std::printf("Build  : [openmxp_b200]\n");
    std::printf("Hash-id: [%s]\n", mxp_version());
    std::printf("BldDate: [%s]\n", __DATE__);
    std::printf("===================================\n");
    std::printf("System : %s\n", a.sys.c_str());
    std::printf("Date   : %s\n", begin.c_str());
    std::printf("JobID  : %d\n", a.jobid);
    std::printf("===================================\n");
    std::printf("N      : %d\n", n);
    std::printf("NB     : %d\n", b);
    std::printf("PMAP   : %s\n", "Row-major");
    std::printf("P      : %d\n", 1);
    std::printf("Q      : %d\n", 1);
    std::printf("PFACT  : %s\n", "Right");
    std::printf("COMM   : %s\n", "on-device");
    std::printf("DEPTH  : %d\n", 1);
    std::printf("U      : %s\n", "transposed form");
    std::printf("L1     : %s\n", "no-transposed form");
    std::printf("TIME(s): %.3f\n", t);
    std::printf("GFLOPS : %.1f\n", flops / t * 1.0e-09);
    std::printf("RESID  : %20.15e\n", resid);
    std::printf("HARNESS: %.9f\n", harness);

    // timer table (timer.hpp:185-208 format) on stderr, from the event-timed phases
    struct Item {
        const char *name;
        double ms;
    } items[] = {{"DIAG_LU", lu.ms_diag_lu},     {"TRSM", lu.ms_trsm},       {"CONV", lu.ms_cast},
                 {"GEMM_UPDATE", lu.ms_schur},   {"IR_GEMV", ir.ms_gemv},    {"IR_TRSV", ir.ms_trsv},
                 {"TOTAL", (double)ms_lu + ms_ir}};
    double misc = ms_lu + ms_ir;
    for (int i = 0; i < 6; ++i) misc -= items[i].ms;
    for (const Item &it : items)
        std::fprintf(stderr, " %-12s : %e sec : %6.2f %%\n", it.name, it.ms / 1e3, 100.0 * it.ms / (ms_lu + ms_ir));
    std::fprintf(stderr, " %-12s : %e sec : %6.2f %%\n", "MISC", misc / 1e3, 100.0 * misc / (ms_lu + ms_ir));
    double gemm_flops = 0.0;
    const int kmul = a.form == MXP_FORM_BF16X2 ? 3 : 1;
    for (int k = 0; k < n / b; ++k) {
        const double m = (double)n - (double)(k + 1) * b;
        gemm_flops += 2.0 * m * m * b * kmul;
    }
    if (lu.ms_schur > 0) std::fprintf(stderr, "GEMM_TOTAL: %f Tflops\n", gemm_flops / (lu.ms_schur / 1e3) * 1e-12);

    mxp_workspace_destroy(ws);
    cudaFree(A);
    cudaFree(d);
    cudaFree(rs);
    cudaFree(rhs);
    cudaFree(x);
    return conv ? 0 : 1;
}
