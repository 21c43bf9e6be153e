/*
 * pfsolve_b200.h -- C ABI of the B200-native Jones-Worland step library.
 *
 * This header is the drop-in boundary for PfSolve's JW path.  It keeps the
 * reference's type names, field names, bitfield values and result codes for
 * the Jones-Worland, dgbmv and block applications, so code written against
 * PfSolve's public API (PfSolve/pfSolve.h) compiles against it for that path:
 *
 *   initializePfSolve  <- PfSolve/pfSolve_AppManagement/pfSolve_InitializeApp.h:1480
 *   PfSolveAppend      <- PfSolve/pfSolve_AppManagement/pfSolve_RunApp.h:80
 *   PfSolveSync        <- PfSolve/pfSolve_AppManagement/pfSolve_RunApp.h:28
 *   deletePfSolve      <- PfSolve/pfSolve_AppManagement/pfSolve_DeleteApp.h:28
 *   PfSolveConfiguration / PfSolveLaunchParams / PfSolveResult
 *                      <- PfSolve/pfSolve_Structs/pfSolve_Structs.h:119-543
 *   app library (checkLibrary_* / addToLibrary_*)
 *                      <- PfSolve/pfSolve_AppCollectionManager.hpp:29-148
 *
 * Only the fields the JW / dgbmv / block applications read are present.
 * The kernels are precompiled for sm_100a; there is no runtime code generation.
 * Entry points marked "extension" have no counterpart in the reference.
 *
 * Everything is plain C: pointers, integers, doubles.  Device buffers are
 * caller-owned; the library never frees them.
 */
#ifndef PFSOLVE_B200_H
#define PFSOLVE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define PFSOLVE_API __attribute__((visibility("default")))
#else
#define PFSOLVE_API
#endif

/* Same types as cuda.h / cuda_runtime_api.h declare (identical redeclaration). */
typedef int CUdevice;
typedef struct CUstream_st* cudaStream_t;

/* jw_control_bitmask: which values come from PfSolveLaunchParams at launch
 * (pfSolve_Structs.h:73-81). */
#define RUNTIME_MSIZE 1
#define RUNTIME_OFFSETM 2
#define RUNTIME_OFFSETV 4
#define RUNTIME_OFFSETSOLUTION 8
#define RUNTIME_INPUTZEROPAD 16
#define RUNTIME_OUTPUTZEROPAD 32
#define RUNTIME_SCALEC 64
#define RUNTIME_INPUTBUFFERSTRIDE 128
#define RUNTIME_OUTPUTBUFFERSTRIDE 256

/* block kernel selector (pfSolve_Structs.h:83-94). */
#define BLOCK_READ_REAL_WRITE_REAL 1
#define BLOCK_READ_COMPLEX_R_WRITE_REAL 2
#define BLOCK_READ_COMPLEX_I_WRITE_REAL 3
#define BLOCK_READ_COMPLEX_STRIDED_WRITE_COMPLEX_PACKED 4
#define BLOCK_READ_REAL_WRITE_COMPLEX_R 5
#define BLOCK_READ_REAL_WRITE_COMPLEX_I 6
#define BLOCK_READ_COMPLEX_PACKED_WRITE_COMPLEX_STRIDED 7
#define BLOCK_ADD_OUTPUTBUFFER_VALUES 20
#define BLOCK_SCALEC 100
#define BLOCK_SCALED 200
#define BLOCK_SCALESPHLAPLA 300
#define BLOCK_SCALESPHLAPLB 400

/* jw_type digits (pfSolve_Structs.h:96-99). */
#define JWT_DISABLE_TRIDIAGONAL_SOLVE 1
#define JWT_DISABLE_MATVECMUL_SOLVE 2
#define JWT_DIAGONAL_MATVECMUL 3
#define JWT_USE_PARALLEL_THOMAS 10

/* Result codes: every code of pfSolve_Structs.h:450-543, same names and
 * numbers (most name backend steps this library never takes; they are kept
 * so that callers' switch statements and getPfSolveErrorString cover them),
 * plus four extension codes. */
typedef enum PfSolveResult {
    PFSOLVE_SUCCESS = 0,
    PFSOLVE_ERROR_MALLOC_FAILED = 1,
    PFSOLVE_ERROR_INSUFFICIENT_CODE_BUFFER = 2,
    PFSOLVE_ERROR_INSUFFICIENT_TEMP_BUFFER = 3,
    PFSOLVE_ERROR_PLAN_NOT_INITIALIZED = 4,
    PFSOLVE_ERROR_NULL_TEMP_PASSED = 5,
    PFSOLVE_ERROR_MATH_FAILED = 6,
    PFSOLVE_ERROR_INVALID_PHYSICAL_DEVICE = 1001,
    PFSOLVE_ERROR_INVALID_DEVICE = 1002,
    PFSOLVE_ERROR_INVALID_QUEUE = 1003,
    PFSOLVE_ERROR_INVALID_COMMAND_POOL = 1004,
    PFSOLVE_ERROR_INVALID_FENCE = 1005,
    PFSOLVE_ERROR_ONLY_FORWARD_FFT_INITIALIZED = 1006,
    PFSOLVE_ERROR_ONLY_INVERSE_FFT_INITIALIZED = 1007,
    PFSOLVE_ERROR_INVALID_CONTEXT = 1008,
    PFSOLVE_ERROR_INVALID_PLATFORM = 1009,
    PFSOLVE_ERROR_ENABLED_saveApplicationToString = 1010,
    PFSOLVE_ERROR_EMPTY_FILE = 1011,
    PFSOLVE_ERROR_EMPTY_FFTdim = 2001,
    PFSOLVE_ERROR_EMPTY_size = 2002,
    PFSOLVE_ERROR_EMPTY_bufferSize = 2003,
    PFSOLVE_ERROR_EMPTY_buffer = 2004,
    PFSOLVE_ERROR_EMPTY_tempBufferSize = 2005,
    PFSOLVE_ERROR_EMPTY_tempBuffer = 2006,
    PFSOLVE_ERROR_EMPTY_inputBufferSize = 2007,
    PFSOLVE_ERROR_EMPTY_inputBuffer = 2008,
    PFSOLVE_ERROR_EMPTY_outputBufferSize = 2009,
    PFSOLVE_ERROR_EMPTY_outputBuffer = 2010,
    PFSOLVE_ERROR_EMPTY_kernelSize = 2011,
    PFSOLVE_ERROR_EMPTY_kernel = 2012,
    PFSOLVE_ERROR_EMPTY_applicationString = 2013,
    PFSOLVE_ERROR_EMPTY_useCustomBluesteinPaddingPattern_arrays = 2014,
    PFSOLVE_ERROR_UNSUPPORTED_RADIX = 3001,
    PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH = 3002,
    PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH_R2C = 3003,
    PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH_DCT = 3004,
    PFSOLVE_ERROR_UNSUPPORTED_FFT_OMIT = 3005,
    PFSOLVE_ERROR_FAILED_TO_ALLOCATE = 4001,
    PFSOLVE_ERROR_FAILED_TO_MAP_MEMORY = 4002,
    PFSOLVE_ERROR_FAILED_TO_ALLOCATE_COMMAND_BUFFERS = 4003,
    PFSOLVE_ERROR_FAILED_TO_BEGIN_COMMAND_BUFFER = 4004,
    PFSOLVE_ERROR_FAILED_TO_END_COMMAND_BUFFER = 4005,
    PFSOLVE_ERROR_FAILED_TO_SUBMIT_QUEUE = 4006,
    PFSOLVE_ERROR_FAILED_TO_WAIT_FOR_FENCES = 4007,
    PFSOLVE_ERROR_FAILED_TO_RESET_FENCES = 4008,
    PFSOLVE_ERROR_FAILED_TO_CREATE_DESCRIPTOR_POOL = 4009,
    PFSOLVE_ERROR_FAILED_TO_CREATE_DESCRIPTOR_SET_LAYOUT = 4010,
    PFSOLVE_ERROR_FAILED_TO_ALLOCATE_DESCRIPTOR_SETS = 4011,
    PFSOLVE_ERROR_FAILED_TO_CREATE_PIPELINE_LAYOUT = 4012,
    PFSOLVE_ERROR_FAILED_SHADER_PREPROCESS = 4013,
    PFSOLVE_ERROR_FAILED_SHADER_PARSE = 4014,
    PFSOLVE_ERROR_FAILED_SHADER_LINK = 4015,
    PFSOLVE_ERROR_FAILED_SPIRV_GENERATE = 4016,
    PFSOLVE_ERROR_FAILED_TO_CREATE_SHADER_MODULE = 4017,
    PFSOLVE_ERROR_FAILED_TO_CREATE_INSTANCE = 4018,
    PFSOLVE_ERROR_FAILED_TO_SETUP_DEBUG_MESSENGER = 4019,
    PFSOLVE_ERROR_FAILED_TO_FIND_PHYSICAL_DEVICE = 4020,
    PFSOLVE_ERROR_FAILED_TO_CREATE_DEVICE = 4021,
    PFSOLVE_ERROR_FAILED_TO_CREATE_FENCE = 4022,
    PFSOLVE_ERROR_FAILED_TO_CREATE_COMMAND_POOL = 4023,
    PFSOLVE_ERROR_FAILED_TO_CREATE_BUFFER = 4024,
    PFSOLVE_ERROR_FAILED_TO_ALLOCATE_MEMORY = 4025,
    PFSOLVE_ERROR_FAILED_TO_BIND_BUFFER_MEMORY = 4026,
    PFSOLVE_ERROR_FAILED_TO_FIND_MEMORY = 4027,
    PFSOLVE_ERROR_FAILED_TO_SYNCHRONIZE = 4028,
    PFSOLVE_ERROR_FAILED_TO_COPY = 4029,
    PFSOLVE_ERROR_FAILED_TO_CREATE_PROGRAM = 4030,
    PFSOLVE_ERROR_FAILED_TO_COMPILE_PROGRAM = 4031,
    PFSOLVE_ERROR_FAILED_TO_GET_CODE_SIZE = 4032,
    PFSOLVE_ERROR_FAILED_TO_GET_CODE = 4033,
    PFSOLVE_ERROR_FAILED_TO_DESTROY_PROGRAM = 4034,
    PFSOLVE_ERROR_FAILED_TO_LOAD_MODULE = 4035,
    PFSOLVE_ERROR_FAILED_TO_GET_FUNCTION = 4036,
    PFSOLVE_ERROR_FAILED_TO_SET_DYNAMIC_SHARED_MEMORY = 4037,
    PFSOLVE_ERROR_FAILED_TO_MODULE_GET_GLOBAL = 4038,
    PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL = 4039,
    PFSOLVE_ERROR_FAILED_TO_EVENT_RECORD = 4040,
    PFSOLVE_ERROR_FAILED_TO_ADD_NAME_EXPRESSION = 4041,
    PFSOLVE_ERROR_FAILED_TO_INITIALIZE = 4042,
    PFSOLVE_ERROR_FAILED_TO_SET_DEVICE_ID = 4043,
    PFSOLVE_ERROR_FAILED_TO_GET_DEVICE = 4044,
    PFSOLVE_ERROR_FAILED_TO_CREATE_CONTEXT = 4045,
    PFSOLVE_ERROR_FAILED_TO_CREATE_PIPELINE = 4046,
    PFSOLVE_ERROR_FAILED_TO_SET_KERNEL_ARG = 4047,
    PFSOLVE_ERROR_FAILED_TO_CREATE_COMMAND_QUEUE = 4048,
    PFSOLVE_ERROR_FAILED_TO_RELEASE_COMMAND_QUEUE = 4049,
    PFSOLVE_ERROR_FAILED_TO_ENUMERATE_DEVICES = 4050,
    PFSOLVE_ERROR_FAILED_TO_GET_ATTRIBUTE = 4051,
    PFSOLVE_ERROR_FAILED_TO_CREATE_EVENT = 4052,
    PFSOLVE_ERROR_FAILED_TO_CREATE_COMMAND_LIST = 4053,
    PFSOLVE_ERROR_FAILED_TO_DESTROY_COMMAND_LIST = 4054,
    PFSOLVE_ERROR_FAILED_TO_SUBMIT_BARRIER = 4055,
    /* extension codes (no counterpart in the reference) */
    PFSOLVE_ERROR_UNSUPPORTED_COMBINATION = 5001, /* parameter combination the reference leaves undefined */
    PFSOLVE_ERROR_INVALID_ARGUMENT = 5002,        /* NULL pointer, negative size, misaligned buffer */
    PFSOLVE_ERROR_CAPACITY = 5003,                /* request exceeds a stated fixed capacity */
    PFSOLVE_ERROR_DEVICE_FAULT = 5004             /* a kernel reported an error status */
} PfSolveResult;

/* Plan-time parameters.  Field names, types and meaning follow
 * PfSolveConfiguration (pfSolve_Structs.h:119-381) for the JW / dgbmv / block
 * applications.  Zero-initialise, then set what you need. */
typedef struct {
    uint64_t FFTdim;      /* must be 1 */
    uint64_t size[3];     /* size[0] = system length (or block row length), size[1] = batch */

    CUdevice* device;     /* device ordinal holder, required */
    cudaStream_t* stream; /* streams to launch on (NULL: default stream) */
    uint64_t num_streams; /* launches rotate over num_streams streams when > 1 */

    uint64_t* bufferSize;       /* optional */
    uint64_t* outputBufferSize; /* optional */
    uint64_t* kernelSize;       /* optional */
    void** buffer;              /* bands (JW, dgbmv) or input (block); may be set at launch */
    void** outputBuffer;        /* right-hand sides, solved in place (JW, dgbmv) or block output */
    void** kernel;              /* temporary buffer (unused by single-upload plans) */

    int upperBanded;      /* 0: lower-banded V / upper M, 1: upper-banded V / lower M, 2: tridiagonal */
    int jw_type;          /* >= 10 selects the JW application; jw_type % 10: 0 matvec+solve,
                             1 matvec only, 2 solve only, 3 diagonal matvec + solve */
    int block;            /* > 0 selects the block application (BLOCK_* sum) */
    int lshift;           /* harmonic degree shift used by the Scale operators */
    int LDA;              /* > 0 selects the dgbmv application: LDA = KL + KU + 1 bands */
    int KU;
    int KL;
    int ALT_dgbmv;        /* dgbmv: drop alternate bands by the reference's rule (pfSolve_Plan_dgbmv.h:100,
                             pfSolve_MatVecMul.h:390); LDA <= 64, not with double-double */
    uint64_t Msplit[3];   /* multi-upload split (accepted, single upload used for M <= 4352) */
    uint64_t performDCT;  /* 2 or 3 selects the DCT application (pfSolve_Structs.h:272): the radial DCT
                             step that feeds the JW chain, DCT-II or DCT-III (FFTW's unnormalized
                             REDFT10 / REDFT01) of size[1]*size[2] rows of size[0] = 2^p points,
                             8 <= size[0] <= 4096, FP64 (doublePrecision); rows are read from buffer at
                             inputBufferStride[0] and written to outputBuffer (or in place to buffer
                             when outputBuffer is NULL) at outputBufferStride[0] (0: size[0]) */

    int64_t jw_control_bitmask; /* RUNTIME_* bits */
    int64_t M_size;
    int64_t offsetM;
    int64_t offsetV;
    int64_t offsetSolution;
    int64_t inputZeropad[2];
    int64_t outputZeropad[2];
    double scaleC;

    /* Precision, in the reference's order (pfSolve_InitAPIParameters.h:148-245):
     * quadDoubleDoublePrecision, quadDoubleDoublePrecisionDoubleMemory, doublePrecision,
     * doublePrecisionFloatMemory; none of them: FP32 storage and arithmetic (the reference's
     * default).  The FP32-storage precisions cover the JW application with M <= 4096 and K = 1
     * (no ALT mode, no mixedPrecisionRefinement), dgbmv, block and fused chains; buffers then
     * hold FP32 values, and offsets and strides count FP32 elements. */
    uint64_t doublePrecision;                       /* FP64 storage and arithmetic */
    uint64_t quadDoubleDoublePrecision;             /* double-double storage and arithmetic */
    uint64_t quadDoubleDoublePrecisionDoubleMemory; /* double-double arithmetic, FP64 storage */
    uint64_t halfPrecision;                         /* not supported: must be 0 */
    uint64_t doublePrecisionFloatMemory;            /* FP64 arithmetic, FP32 storage */

    uint64_t inputBufferStride[3];
    uint64_t outputBufferStride[3];
    uint64_t isInputFormatted;
    uint64_t isOutputFormatted;

    uint64_t keepShaderCode;    /* accepted; there is no generated code to print */
    uint64_t printMemoryLayout; /* accepted */
    int disableCaching;         /* accepted; plans are never cached on disk */
    uint64_t disableSetLocale;  /* accepted */
    uint64_t useUint64;         /* accepted; addressing is always 64-bit */

    int numConsecutiveJWIterations; /* K consecutive steps in one kernel, 1..8: upperBanded 0/1 with
                                       jw_type % 10 in {0, 1, 2}; upperBanded 2 with K = 2
                                       (pfSolve_JonesWorland.h:108-374); FP64 only */
    int useMultipleInputBuffers;    /* >= K: bands of step k in buffer[k]; 0 or 1: every step reads
                                       buffer[0] at its own offsets (pfSolve_Transfers.h:250-265) */

    /* --- extensions (0 keeps the reference behaviour) --- */
    int mixedPrecisionRefinement; /* 1..3 with doublePrecision: FP32 factor-solve plus this many
                                     FP64 residual refinement sweeps, FP64 storage (0: plain FP64) */
    int rowsPerThread;            /* 0: autotuned; else 2, 4, 8, 16 or 32 (32: streaming kernel only) */
    int kernelPath;               /* 0: streaming kernel wherever a launch allows it, else the group
                                     kernel (long systems: two passes, with the single pass for
                                     launches whose rows are not 16-byte aligned); 1: group kernel
                                     only; 2: long systems on the
                                     cluster kernel (M <= 16384); 3: long systems in two passes only (no
                                     waits between CTAs); 4: long systems in the single pass only */
    int stagingBuffers;           /* streaming kernel: TMA staging buffers per group of warps, 2..4, so
                                     that up to stagingBuffers - 1 systems' loads are in flight while
                                     one is solved (0: 2, or 3 for FP32 storage and arithmetic where
                                     they fit beside as many groups); more buffers can mean fewer
                                     groups per CTA */
} PfSolveConfiguration;

/* Launch-time values (pfSolve_Structs.h:383-449). */
typedef struct {
    void** buffer;       /* bands / block input; NULL keeps the plan's */
    void** outputBuffer; /* right-hand sides / block output; NULL keeps the plan's */
    void** kernel;

    uint64_t M_size;
    uint64_t offsetM;
    uint64_t offsetV;
    uint64_t offsetSolution;
    uint64_t inputZeropad[2];
    uint64_t outputZeropad[2];
    long double scaleC;
    uint64_t inputBufferStride;
    uint64_t outputBufferStride;
    uint64_t batchSize; /* > 0 replaces size[1] for this and later launches */
} PfSolveLaunchParams;

/* Opaque plan state lives behind `internal`; `configuration` is the copy
 * initializePfSolve validated (pfSolve_Structs.h:1292-1341 holds the
 * reference's larger struct). */
typedef struct PfSolveApplication {
    PfSolveConfiguration configuration;
    void* internal;
} PfSolveApplication;

/* Validate `configuration` (passed by value, as in the reference), pick the
 * kernel variant and launch shape, and query the device.  On failure the app
 * is released and the error returned. */
PFSOLVE_API PfSolveResult initializePfSolve(PfSolveApplication* app, PfSolveConfiguration configuration);

/* Enqueue one application launch on the plan's stream; never synchronises.
 * `inverse` is ignored, as in the reference. */
PFSOLVE_API PfSolveResult PfSolveAppend(PfSolveApplication* app, int inverse, PfSolveLaunchParams* launchParams);

/* Wait for the plan's streams when num_streams > 1 (no-op otherwise). */
PFSOLVE_API PfSolveResult PfSolveSync(PfSolveApplication* app);

/* Release the plan's host and device state (never the user's buffers). */
PFSOLVE_API void deletePfSolve(PfSolveApplication* app);

/* Name of a result code, as the reference's helper of the same name
 * (pfSolve_Structs/pfSolve_Structs.h:545): every code declared above has its
 * own name; other values give "PFSOLVE_ERROR_UNKNOWN". */
PFSOLVE_API const char* getPfSolveErrorString(PfSolveResult result);
/* The reference's version value (pfSolve.h:101-103): its source writes it as
 * the literal 00102 ("X.XX.XX format"), which C reads as octal, so the value
 * is 66. */
PFSOLVE_API int PfSolveGetVersion(void);

/* ---- App library (kernel reuse cache), pfSolve_AppCollectionManager.hpp ---- */
typedef struct PfSolve_MapKey_JonesWorland {
    int64_t size[2];
    int64_t upperBanded;
    int64_t outputBufferStride;
    int64_t type;
} PfSolve_MapKey_JonesWorland;
typedef struct PfSolve_MapKey_dgbmv {
    int64_t size[2];
    int64_t outputBufferStride;
    int64_t LDA;
    int64_t KU;
    int64_t KL;
} PfSolve_MapKey_dgbmv;
typedef struct PfSolve_MapKey_block {
    int64_t size[2];
    int64_t inputBufferStride;
    int64_t outputBufferStride;
    int64_t type;
    int64_t lshift;
} PfSolve_MapKey_block;

typedef struct PfSolve_AppLibrary PfSolve_AppLibrary;

PFSOLVE_API PfSolve_AppLibrary* PfSolveAppLibraryCreate(void);                 /* extension: C handle */
PFSOLVE_API void PfSolveAppLibraryDestroy(PfSolve_AppLibrary* lib);            /* extension: deletes the apps it holds */
PFSOLVE_API PfSolveResult checkLibrary_JonesWorland(PfSolve_AppLibrary* lib, PfSolve_MapKey_JonesWorland key, PfSolveApplication** app);
PFSOLVE_API PfSolveResult addToLibrary_JonesWorland(PfSolve_AppLibrary* lib, PfSolve_MapKey_JonesWorland key, PfSolveApplication* app);
PFSOLVE_API PfSolveResult checkLibrary_dgbmv(PfSolve_AppLibrary* lib, PfSolve_MapKey_dgbmv key, PfSolveApplication** app);
PFSOLVE_API PfSolveResult addToLibrary_dgbmv(PfSolve_AppLibrary* lib, PfSolve_MapKey_dgbmv key, PfSolveApplication* app);
PFSOLVE_API PfSolveResult checkLibrary_block(PfSolve_AppLibrary* lib, PfSolve_MapKey_block key, PfSolveApplication** app);
PFSOLVE_API PfSolveResult addToLibrary_block(PfSolve_AppLibrary* lib, PfSolve_MapKey_block key, PfSolveApplication* app);

/* ---- Fused chain (extension) ----
 * Runs apps[0..n-1] as if appended one after the other on the same data, in
 * one kernel when the chain is [dgbmv] -> JW -> [block] over the same systems.
 * Intermediate results are not written back to memory.  Returns
 * PFSOLVE_ERROR_UNSUPPORTED_COMBINATION when the chain cannot be fused and
 * `allowUnfused` is 0; with allowUnfused the apps run one by one. */
PFSOLVE_API PfSolveResult PfSolveAppendChain(PfSolveApplication** apps, PfSolveLaunchParams** launchParams, int n,
                                 int allowUnfused);

/* ---- Uneven batch (extension) ----
 * One JW step over many groups of systems of different sizes (one group per
 * harmonic degree of a spectral timestep), in ONE persistent launch: groups
 * of warps take (entry, system range) items from a device work queue,
 * largest first, and refactor the matrix when the entry changes.  The step is
 * the chain [dgbmv] -> JW -> [block] of the apps with the same fields.
 * Every entry uses plan-time band offsets: JW bands at 0, M, 2M of `bands`
 * (reference register-major order for its own M), dgbmv bands band-major.
 * Two kernels: the group kernel (a group of warps per system, rowsPerThread
 * rows per thread) and the sweep kernel (one complex system per lane, its
 * rows in sequence, a warp per item of 32 systems).  sweepRows = 8 or 16
 * asks for the sweep kernel with that many rows per staged chunk
 * (PFSOLVE_ERROR_UNSUPPORTED_COMBINATION where the batch does not allow it).
 * With rowsPerThread, systemsPerItem and sweepRows all 0 the sweep kernel runs
 * wherever the batch allows it:
 * FP64, a bidiagonal (or no) solve, the fused V*A within rows i-1..i+1, block
 * 7 (XXII in, packed complex out) without accumulation, and every entry's
 * output 16-byte aligned and disjoint from its input. */
typedef struct {
    int64_t M;               /* rows of this entry's systems (<= 4096) */
    int64_t nsys;            /* systems (complex ones count once) */
    const void* bands;       /* JW bands of this entry (device) */
    const void* dgbmvBands;  /* band-major matrix of the fused dgbmv (device), or NULL */
    const void* input;       /* system y: input + y*inputStride (XXII: rows 2y and 2y+1) */
    void* output;            /* system y: output + y*outputStride (packed complex: in complex elements) */
    int64_t inputStride;
    int64_t outputStride;
    int lshift;              /* Scale operator's harmonic degree */
    double scaleS;           /* Scale operator's s (its scaleC) */
    double scaleC;           /* JW scaleC on solution row 0 */
} PfSolveBatchEntry;

typedef struct {
    int upperBanded;              /* JW step of every entry */
    int jw_type;
    int LDA, KU, KL;              /* fused dgbmv (LDA = 0: none) */
    int block;                    /* fused block epilogue: 0, 1 (real) or 7 (XXII -> packed) plus
                                     100 * Scale kind (BLOCK_SCALEC ... BLOCK_SCALESPHLAPLB) */
    int mixedPrecisionRefinement; /* as in PfSolveConfiguration */
    int rowsPerThread;            /* 0: default / autotuned */
    int systemsPerItem;           /* work-queue item size (0: default / autotuned) */
    int sweepRows;                /* sweep kernel with chunks of 8 or 16 rows (0: default / autotuned) */
} PfSolveBatchDesc;

typedef struct PfSolveBatch PfSolveBatch;

/* Build a batch plan: copies the entry descriptors and the work list to the
 * device (owned by the plan). */
PFSOLVE_API PfSolveResult PfSolveBatchCreate(PfSolveBatch** batch, CUdevice device, const PfSolveBatchDesc* desc,
                                             const PfSolveBatchEntry* entries, int nentries);
/* Enqueue the whole batch: a work-queue reset and one persistent kernel (or
 * the captured graph of exactly that). */
PFSOLVE_API PfSolveResult PfSolveBatchAppend(PfSolveBatch* batch, cudaStream_t stream);
/* Capture the batch's launch into a CUDA graph on `stream` (a non-default
 * stream); later PfSolveBatchAppend calls launch the graph. */
PFSOLVE_API PfSolveResult PfSolveBatchCaptureGraph(PfSolveBatch* batch, cudaStream_t stream);
/* Time every compiled rows-per-thread / item-size candidate of the group
 * kernel, and the sweep kernel where the batch allows it, on the batch's own
 * buffers (`iterations` launches each) and keep the fastest; drops a
 * captured graph.  Entries must be out of place (input != output). */
PFSOLVE_API PfSolveResult PfSolveBatchAutotune(PfSolveBatch* batch, cudaStream_t stream, int iterations);
/* Chosen shape: rows per thread, warps per system, systems per item, work
 * items, and the autotuner's best time (ms, 0 when not tuned).  Rows per
 * thread and warps per system 0: the sweep kernel. */
PFSOLVE_API PfSolveResult PfSolveBatchGetShape(const PfSolveBatch* batch, int* rowsPerThread, int* warpsPerSystem,
                                               int* systemsPerItem, int* items, double* tunedMs);
/* The sweep kernel's shape: rows per staged chunk, chunk buffers per warp and
 * warps per CTA (all 0 when the batch runs the group kernel). */
PFSOLVE_API PfSolveResult PfSolveBatchGetSweepShape(const PfSolveBatch* batch, int* rowsPerChunk, int* buffers,
                                                    int* warpsPerCTA);
PFSOLVE_API void PfSolveBatchDestroy(PfSolveBatch* batch);

/* One uneven batch, as PfSolveBatchCreate + PfSolveBatchAppend +
 * PfSolveBatchDestroy, that allocates nothing: no cudaMalloc, no cudaFree,
 * no host heap (the work list is sorted in place in fixed host arrays).
 * For callers that must not reach the device allocator during
 * their time loop -- code whose device memory is all owned by its own pool,
 * or which cannot afford the implicit device synchronisation and the failure
 * modes of cudaMalloc.  No counterpart in the reference.
 * The work list, the entry descriptors and the work counter live in one fixed
 * device array inside the library, sized for PFSOLVE_NOALLOC_MAX_ENTRIES
 * entries and PFSOLVE_NOALLOC_MAX_ITEMS work items (ceil(nsys /
 * systemsPerItem) per entry, systemsPerItem 0 meaning 64); larger calls return
 * PFSOLVE_ERROR_CAPACITY.  It runs the group kernel only (sweepRows must be
 * 0).  The work counter must start at zero: each call
 * clears it on `stream` before its launch.  All calls share the array, so two
 * calls whose work overlaps in time (on other streams or from other threads)
 * race; serialise them.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress); make that call before any stream
 * capture on the device.  The descriptors reach the device by
 * cudaMemcpyAsync from the library's fixed host arrays, which are ordinary
 * (pageable) memory: the call returns once the driver has staged them, so it
 * may block the host for that copy (never for the device's queued work).
 * The next call rewrites those host arrays, so a call on a stream that is
 * being captured returns PFSOLVE_ERROR_INVALID_ARGUMENT and enqueues nothing;
 * do not issue it under stream capture.
 * The caller's current device is the same on return as on entry.  Results
 * equal PfSolveBatchAppend's for the same descriptor, rows per thread and
 * systems per item. */
#define PFSOLVE_NOALLOC_MAX_ENTRIES 1024
#define PFSOLVE_NOALLOC_MAX_ITEMS 16384
PFSOLVE_API PfSolveResult PfSolveBatchAppendNoAlloc(CUdevice device, const PfSolveBatchDesc* desc,
                                                   const PfSolveBatchEntry* entries, int nentries,
                                                   cudaStream_t stream);

/* Number of kernel launches this library has enqueued since load (all apps). */
PFSOLVE_API uint64_t PfSolveLaunchCount(void);

/* Status of the bounded completion waits inside this library's kernels on
 * the current device since the previous call: PFSOLVE_SUCCESS, or
 * PFSOLVE_ERROR_DEVICE_FAULT when a wait ran out and a kernel stopped early
 * (its output is incomplete).  Synchronises with the device.  No counterpart
 * in the reference, whose generated kernels have no such waits. */
PFSOLVE_API PfSolveResult PfSolveGetDeviceStatus(void);

/* Kernel shape a JW or dgbmv plan chose: streaming = 1 when its launches use
 * the TMA-staged streaming kernel wherever their buffers allow it, with
 * rowsPerThread x warpsPerSystem rows per group and groupsPerCTA groups;
 * streaming = 0: the group kernel's shape; streaming = 2: long systems
 * (M > 4096), one thread-block cluster per system, warpsPerSystem warps over
 * the cluster's CTAs; streaming = 3: the K-step kernel
 * (numConsecutiveJWIterations > 1); streaming = 4: K bidiagonal steps with one
 * system per lane in one sweep wherever a launch's buffers allow it
 * (16-byte-aligned rows, stride >= the rows written, full output window;
 * groupsPerCTA = warps per CTA), else the K-step kernel; streaming = 5: long
 * systems (M > 4096) over slices of 32 x warpsPerSystem x rowsPerThread rows,
 * groupsPerCTA systems in flight per CTA: two passes with no waits between
 * CTAs (the default, and kernelPath 3), or a single cooperative pass whose
 * CTAs wait (bounded) for the other slices of each system (kernelPath 4, and
 * a two-pass plan's launches whose rows are not 16-byte aligned); a last
 * partial chunk of rowsPerThread rows moves by plain loads and stores; the
 * plan holds a record of 64 bytes
 * and a 4-byte flag per system and slice, and every slice's coefficient
 * table.
 * No counterpart in the reference. */
PFSOLVE_API PfSolveResult PfSolveGetShape(const PfSolveApplication* app, int* streaming, int* rowsPerThread,
                                          int* warpsPerSystem, int* groupsPerCTA);
/* Launches that ran on the streaming kernel since load (all apps). */
PFSOLVE_API uint64_t PfSolveStreamingLaunchCount(void);

/* The kernel instance of the most recent launch this library enqueued from
 * the calling thread (PfSolveAppend, PfSolveAppendChain), so that a caller
 * or a test can tell which compiled kernel ran.  No counterpart in the
 * reference. */
enum {
    PFSOLVE_KERNEL_NONE = 0,      /* no launch yet on this thread */
    PFSOLVE_KERNEL_GROUP = 1,     /* jw_step_kernel: a group of warps per system, cp.async staging */
    PFSOLVE_KERNEL_STREAMING = 2, /* jw_stream_kernel: whole systems staged by TMA */
    PFSOLVE_KERNEL_LONG = 3,      /* jw_long_kernel: long systems in two passes over slices */
    PFSOLVE_KERNEL_CLUSTER = 4,   /* jw_cluster_kernel: one thread-block cluster per long system */
    PFSOLVE_KERNEL_STEPS = 5,     /* jw_steps_kernel: K consecutive steps */
    PFSOLVE_KERNEL_STEPS_SWEEP = 6, /* jw_steps_seq_kernel: K bidiagonal steps, one system per lane */
    PFSOLVE_KERNEL_DGBMV = 7,     /* dgbmv_generic_kernel: band matrices wider than two bands a side */
    PFSOLVE_KERNEL_BLOCK = 8,     /* block_kernel */
    PFSOLVE_KERNEL_DCT = 9        /* dct_kernel: the DCT step (performDCT 2 or 3) */
};
typedef struct {
    int kernel;         /* PFSOLVE_KERNEL_* */
    int rowsPerThread;  /* 0 where the kernel has no such parameter */
    int warpsPerSystem;
    int groupsPerCTA;
    int bandsBelow;     /* KL of the fused matvec weights (JW matvec and dgbmv together) */
    int bandsAbove;     /* KU */
    int solve;          /* 0 none, 1 unit lower, 2 unit upper, 3 unit tridiagonal */
    int layoutIn;       /* 0 real rows, 1 complex XXII (real rows, then imaginary rows), 2 packed complex */
    int layoutOut;
    int scale;          /* a fused Scale operator (block 1xx..4xx) */
    int precision;      /* 0 FP64, 1 FP32 solve + FP64 refinement, 2 double-double storage, 3 double-double on
                           FP64 storage, 4 FP32, 5 FP64 arithmetic on FP32 storage */
    int alt;            /* ALT stride-2 mode */
    int64_t gridCTAs;   /* CTAs of the (last) kernel of the launch */
} PfSolveLaunchInfo;
PFSOLVE_API PfSolveResult PfSolveGetLastLaunch(PfSolveLaunchInfo* info);

/* ---- Serving engine.  No counterpart in the reference (whose callers drive
 * one application at a time): JW-step requests of mixed size and precision are
 * queued, admitted while the bytes of the requests on the device stay within
 * an HBM budget, batched as they arrive and run on several streams at once, so
 * requests that arrive while others run start without waiting for them.
 * Operators (bands) are registered once and stay resident on the device. */
typedef struct PfSolveServer PfSolveServer;

typedef struct {
    int device;
    uint64_t hbmBudgetBytes;  /* in-flight request bytes (inputs + outputs) admitted at once */
    int streams;              /* batches on the device at once (1..16) */
    int maxBatchRequests;     /* requests per batch (1..256) */
    int refineSweeps;         /* FP64 refinement sweeps of mixed-precision requests (1..3) */
} PfSolveServerDesc;

enum { PFSOLVE_SERVE_MIXED = 1, PFSOLVE_SERVE_DD = 2, PFSOLVE_SERVE_DD_FP64MEM = 3 };

typedef struct {
    int op;              /* operator id from PfSolveServerAddOperator */
    int precision;       /* PFSOLVE_SERVE_*: FP32 solve + FP64 refinement (FP64 storage), double-double
                            storage ({hi, lo} per value), double-double arithmetic on FP64 storage */
    int64_t nrhs;        /* right-hand sides (systems) */
    const void* input;   /* device, systems `stride` values apart */
    void* output;        /* device; may equal input */
    int64_t stride;      /* values between consecutive systems (0: M) */
    double scaleC;       /* multiplies solution row 0 */
    cudaStream_t stream; /* the caller's stream that writes `input` (NULL: the legacy default stream).  The
                            server's streams do not synchronise with the caller's, so Submit records an event
                            on this stream and the request's kernel waits for it: work the caller enqueued on
                            it before Submit (writing the input, clearing the output) comes first. */
    int inputReady;      /* 1: skip that wait -- the caller guarantees that nothing still pending on the
                            device writes `input` or `output` (e.g. it synchronised) */
} PfSolveRequest;

typedef struct {
    uint64_t submitted, completed, batches, rhs;
    uint64_t peakInflightBytes;
    double p50Ms, p99Ms, maxMs;  /* submit -> completion on the GPU, over completed requests */
    double p99QueueMs;           /* submit -> launch enqueued (queueing and admission) */
    double p99DeviceMs;          /* launch enqueued -> completion (device time and completion signal) */
} PfSolveServerStats;

PFSOLVE_API PfSolveResult PfSolveServerCreate(PfSolveServer** server, const PfSolveServerDesc* desc);
/* Register an operator: JW bands in the reference's layout (3*M doubles, device
 * memory that stays valid while the server lives), upperBanded / jw_type as in
 * PfSolveConfiguration.  A double-double copy is made on the device. */
PFSOLVE_API PfSolveResult PfSolveServerAddOperator(PfSolveServer* server, int64_t M, const double* bands,
                                                   int upperBanded, int jw_type, int* opId);
/* Queue a request; returns at once (after recording the ordering event on
 * request->stream unless inputReady).  PFSOLVE_ERROR_CAPACITY when the
 * request alone exceeds the HBM budget.  The output is complete, and visible
 * to any later work of the caller, once PfSolveServerWait returns. */
PFSOLVE_API PfSolveResult PfSolveServerSubmit(PfSolveServer* server, const PfSolveRequest* request,
                                              uint64_t* ticket);
/* Block until the request is done; its latency (ms) when latencyMs != NULL.
 * Returns the request's status: PFSOLVE_SUCCESS, or the launch error that
 * left its output unwritten.  Each ticket is waited on once. */
PFSOLVE_API PfSolveResult PfSolveServerWait(PfSolveServer* server, uint64_t ticket, double* latencyMs);
PFSOLVE_API PfSolveResult PfSolveServerGetStats(PfSolveServer* server, PfSolveServerStats* stats);
/* Drain every queued request, then free the server. */
PFSOLVE_API void PfSolveServerDestroy(PfSolveServer* server);

#ifdef __cplusplus
}
#endif
#endif /* PFSOLVE_B200_H */
