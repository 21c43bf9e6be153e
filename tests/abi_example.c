/* jw_step.c: one FP64 JW step (upperBanded 2, jw_type 13) on B systems in place.
 * cc -std=c11 -I include jw_step.c -L pfsolve_b200 -lpfsolve_b200 -Wl,-rpath,pfsolve_b200 */
#include <string.h>
#include "pfsolve_b200.h"

int jw_step(double* d_bands, double* d_rhs, int64_t M, uint64_t B, cudaStream_t stream)
{
    PfSolveApplication app;
    PfSolveConfiguration cfg;
    memset(&cfg, 0, sizeof(cfg));
    CUdevice dev = 0;
    cfg.FFTdim = 1;
    cfg.size[0] = (uint64_t)M;
    cfg.size[1] = B;
    cfg.M_size = M;
    cfg.device = &dev;
    cfg.stream = &stream;
    cfg.num_streams = 1;
    cfg.doublePrecision = 1;
    cfg.upperBanded = 2;
    cfg.jw_type = 13;
    cfg.scaleC = 1.0; /* a zero-initialised config has scaleC = 0, which zeroes row 0 */
    cfg.buffer = (void**)&d_bands;
    cfg.outputBuffer = (void**)&d_rhs;
    PfSolveResult r = initializePfSolve(&app, cfg);
    if (r != PFSOLVE_SUCCESS) return (int)r;
    PfSolveLaunchParams lp;
    memset(&lp, 0, sizeof(lp));
    r = PfSolveAppend(&app, 0, &lp);
    deletePfSolve(&app);
    return (int)r;
}
