// ref_harness.cpp -- drives the UNMODIFIED PfSolve library (header-only, compiled
// from the reference's own sources by oracle/Makefile into oracle/_ref/) through
// its public C API: initializePfSolve -> PfSolveAppend -> deletePfSolve.
//
// TEST INFRASTRUCTURE ONLY.  It produces the reference's own GPU outputs for
// seeded inputs (golden vectors that pin the C oracle) and times the reference
// kernels on the same GPU.  The product never links or runs it.
//
// Usage: pfsolve_ref <case_dir>
//   <case_dir>/params.txt   key=value lines (see parse below)
//   <case_dir>/bands.bin    band buffer (raw, storage precision), or
//   <case_dir>/bands_<k>.bin one buffer per step when useMultipleInputBuffers > 1
//   <case_dir>/rhs.bin      output/RHS buffer (raw, storage precision), in place
//   <case_dir>/in.bin       block kernel only: its input buffer
// Writes <case_dir>/out.bin (the RHS/output buffer after one launch) and,
// when iters > 0, <case_dir>/time.txt (mean ms per PfSolveAppend over `iters`
// back-to-back launches on one stream, CUDA events).
#include "pfSolve.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include <csignal>
#include <execinfo.h>
#include <unistd.h>

// Host crash report: the phase the harness was in and the return addresses
// (offsets into this binary, for addr2line), written to stderr.
static const char* volatile g_phase = "setup";

static void on_crash(int sig)
{
    void* frames[48];
    int n = backtrace(frames, 48);
    dprintf(2, "signal %d in phase %s\n", sig, g_phase);
    backtrace_symbols_fd(frames, n, 2);
    _exit(128 + sig);
}

static std::map<std::string, std::string> read_params(const std::string& path)
{
    std::map<std::string, std::string> kv;
    FILE* f = fopen(path.c_str(), "r");
    if (!f) return kv;
    char line[512];
    while (fgets(line, sizeof line, f)) {
        char* eq = strchr(line, '=');
        if (!eq) continue;
        *eq = 0;
        std::string k(line), v(eq + 1);
        while (!v.empty() && (v.back() == '\n' || v.back() == '\r')) v.pop_back();
        kv[k] = v;
    }
    fclose(f);
    return kv;
}

static std::vector<char> read_file(const std::string& path)
{
    std::vector<char> b;
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return b;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    b.resize((size_t)n);
    if (n > 0 && fread(b.data(), 1, (size_t)n, f) != (size_t)n) b.clear();
    fclose(f);
    return b;
}

int main(int argc, char** argv)
{
    if (argc < 2) { fprintf(stderr, "usage: %s <case_dir>\n", argv[0]); return 2; }
    std::string dir = argv[1];
    signal(SIGSEGV, on_crash);
    signal(SIGABRT, on_crash);
    auto kv = read_params(dir + "/params.txt");
    auto I = [&](const char* k, long long d) { return kv.count(k) ? atoll(kv[k].c_str()) : d; };
    auto D = [&](const char* k, double d) { return kv.count(k) ? atof(kv[k].c_str()) : d; };

    if (cuInit(0) != CUDA_SUCCESS) { fprintf(stderr, "cuInit failed\n"); return 3; }
    if (cudaSetDevice(0) != cudaSuccess) { fprintf(stderr, "cudaSetDevice failed\n"); return 3; }
    CUdevice dev;
    cuDeviceGet(&dev, 0);
    cudaFree(0);  // create the primary context through the runtime

    const int nbuf = (int)I("useMultipleInputBuffers", 1);
    std::vector<std::vector<char>> step_bands;
    if (nbuf > 1)
        for (int k = 0; k < nbuf; k++) step_bands.push_back(read_file(dir + "/bands_" + std::to_string(k) + ".bin"));
    std::vector<char> bands = nbuf > 1 ? step_bands[0] : read_file(dir + "/bands.bin");
    std::vector<char> rhs = read_file(dir + "/rhs.bin");
    std::vector<char> inb = read_file(dir + "/in.bin");
    // Timing cases may omit rhs.bin: `rhs_bytes` zero-filled device bytes instead.
    const long long rhs_bytes = I("rhs_bytes", 0);
    if (rhs.empty() && rhs_bytes <= 0) { fprintf(stderr, "missing rhs.bin\n"); return 2; }

    void* d_bands = nullptr;
    void* d_rhs = nullptr;
    void* d_in = nullptr;
    void* d_tmp = nullptr;
    uint64_t bandsSize = bands.empty() ? 16 : bands.size();
    uint64_t rhsSize = rhs.empty() ? (uint64_t)rhs_bytes : rhs.size();
    uint64_t inSize = inb.empty() ? 16 : inb.size();
    if (cudaMalloc(&d_bands, bandsSize) || cudaMalloc(&d_rhs, rhsSize) || cudaMalloc(&d_in, inSize) ||
        cudaMalloc(&d_tmp, rhsSize)) {
        fprintf(stderr, "cudaMalloc failed\n");
        return 4;
    }
    if (!bands.empty()) cudaMemcpy(d_bands, bands.data(), bands.size(), cudaMemcpyHostToDevice);
    if (rhs.empty()) cudaMemset(d_rhs, 0, rhsSize);
    else cudaMemcpy(d_rhs, rhs.data(), rhs.size(), cudaMemcpyHostToDevice);
    if (!inb.empty()) cudaMemcpy(d_in, inb.data(), inb.size(), cudaMemcpyHostToDevice);

    PfSolveConfiguration cfg = {};
    PfSolveApplication app = {};
    cfg.FFTdim = 1;
    cfg.M_size = I("M", 0);
    cfg.size[0] = I("size0", cfg.M_size);
    cfg.size[1] = I("size1", 1);
    cfg.size[2] = 1;
    cfg.doublePrecision = I("doublePrecision", 1);
    cfg.quadDoubleDoublePrecision = I("quadDoubleDoublePrecision", 0);
    cfg.quadDoubleDoublePrecisionDoubleMemory = I("quadDoubleDoublePrecisionDoubleMemory", 0);
    cfg.doublePrecisionFloatMemory = I("doublePrecisionFloatMemory", 0);
    cfg.isOutputFormatted = 1;
    cfg.jw_type = (int)I("jw_type", 0);
    cfg.upperBanded = (int)I("upperBanded", 0);
    cfg.jw_control_bitmask = I("bitmask", 0);
    cfg.numConsecutiveJWIterations = (int)I("K", 1);
    cfg.useMultipleInputBuffers = (int)I("useMultipleInputBuffers", 1);
    cfg.offsetM = I("cfg_offsetM", 0);
    cfg.offsetV = I("cfg_offsetV", 0);
    cfg.offsetSolution = I("cfg_offsetSolution", 0);
    cfg.inputZeropad[0] = I("cfg_iz0", 0);
    cfg.inputZeropad[1] = I("cfg_iz1", 0);
    cfg.outputZeropad[0] = I("cfg_oz0", 0);
    cfg.outputZeropad[1] = I("cfg_oz1", 0);
    cfg.scaleC = D("cfg_scaleC", 1.0);
    cfg.inputBufferStride[0] = I("cfg_inputBufferStride", cfg.size[0]);
    cfg.outputBufferStride[0] = I("cfg_outputBufferStride", cfg.size[0]);
    cfg.LDA = (int)I("LDA", 0);
    cfg.KU = (int)I("KU", 0);
    cfg.KL = (int)I("KL", 0);
    cfg.ALT_dgbmv = (int)I("ALT_dgbmv", 0);
    cfg.block = (int)I("block", 0);
    cfg.lshift = (int)I("lshift", 0);
    cfg.disableCaching = 1;  // no kernel cache files are written or read
    // code-generation buffers (0 keeps the reference's defaults: 4 000 000 and
    // 5 000 chars); its double-double kernels need a larger intermediate buffer
    cfg.maxCodeLength = I("maxCodeLength", 0);
    cfg.maxTempLength = I("maxTempLength", 0);
    cfg.device = &dev;

    void* bufArr[16] = {cfg.block ? d_in : d_bands};
    if (nbuf > 16) { fprintf(stderr, "at most 16 input buffers\n"); return 2; }
    for (int k = 1; k < nbuf; k++) {
        const std::vector<char>& b = step_bands[k];
        if (b.empty() || cudaMalloc(&bufArr[k], b.size())) { fprintf(stderr, "bands_%d\n", k); return 4; }
        cudaMemcpy(bufArr[k], b.data(), b.size(), cudaMemcpyHostToDevice);
    }
    void* outArr[1] = {d_rhs};
    void* tmpArr[1] = {d_tmp};
    uint64_t bufSizeArr[1] = {cfg.block ? inSize : bandsSize};
    uint64_t outSizeArr[1] = {rhsSize};
    cfg.buffer = bufArr;
    cfg.outputBuffer = outArr;
    cfg.kernel = tmpArr;
    cfg.bufferSize = bufSizeArr;
    cfg.outputBufferSize = outSizeArr;
    cfg.kernelSize = outSizeArr;

    g_phase = "initializePfSolve";
    PfSolveResult r = initializePfSolve(&app, cfg);
    if (r != PFSOLVE_SUCCESS) { fprintf(stderr, "initializePfSolve: %d\n", (int)r); return 10; }

    PfSolveLaunchParams lp = {};
    lp.buffer = bufArr;
    lp.outputBuffer = outArr;
    lp.kernel = tmpArr;
    lp.offsetM = I("run_offsetM", 0);
    lp.offsetV = I("run_offsetV", 0);
    lp.offsetSolution = I("run_offsetSolution", 0);
    lp.inputZeropad[0] = I("run_iz0", 0);
    lp.inputZeropad[1] = I("run_iz1", cfg.M_size);
    lp.outputZeropad[0] = I("run_oz0", 0);
    lp.outputZeropad[1] = I("run_oz1", cfg.M_size);
    lp.scaleC = D("run_scaleC", 1.0);
    lp.inputBufferStride = I("run_inputBufferStride", cfg.size[0]);
    lp.outputBufferStride = I("run_outputBufferStride", cfg.size[0]);

    g_phase = "PfSolveAppend";
    r = PfSolveAppend(&app, 0, &lp);
    if (r != PFSOLVE_SUCCESS) { fprintf(stderr, "PfSolveAppend: %d\n", (int)r); return 11; }
    g_phase = "after launch";
    cudaError_t ce = cudaDeviceSynchronize();
    if (ce != cudaSuccess) { fprintf(stderr, "sync: %s\n", cudaGetErrorString(ce)); return 12; }
    if (!rhs.empty()) {
        std::vector<char> out(rhsSize);
        cudaMemcpy(out.data(), d_rhs, rhsSize, cudaMemcpyDeviceToHost);
        FILE* fo = fopen((dir + "/out.bin").c_str(), "wb");
        if (!fo) return 13;
        fwrite(out.data(), 1, out.size(), fo);
        fclose(fo);
    }

    long long iters = I("iters", 0);
    if (iters > 0) {
        for (int w = 0; w < 3; w++) PfSolveAppend(&app, 0, &lp);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, 0);
        for (long long it = 0; it < iters; it++) PfSolveAppend(&app, 0, &lp);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        FILE* ft = fopen((dir + "/time.txt").c_str(), "w");
        if (ft) { fprintf(ft, "%.6f\n", ms / (double)iters); fclose(ft); }
    }
    deletePfSolve(&app);
    for (int k = 1; k < nbuf; k++) cudaFree(bufArr[k]);
    cudaFree(d_bands);
    cudaFree(d_rhs);
    cudaFree(d_in);
    cudaFree(d_tmp);
    return 0;
}
