// Kernel argument structs and launcher declarations shared by fg_kernels.cu and fg_solver.cu.
#pragma once
#include "fg_device.cuh"

namespace fg {

// Cell-ordered (renumbered) device mesh.  Per-slot arrays are cell-major: a[c * nSlots + k], so
// the lanes that work on the faces of one cell read contiguous words.
template <typename T>
struct DevMesh {
    int n;              // cells with records (W, G): own cells, then the ghosts of a partitioned mesh
    int nU;             // own cells: the first nU cells carry a state (U, U0, RHS rows) and are updated
    int nG;             // cells with gradients: own cells, then a part's first-layer ghosts
    int nFEval;         // faces the face kernel evaluates (those touching an own cell) come first
    int nSlots;         // max faces per cell
    const int32_t *nbr;   // neighbour cell, or -bc (1..5) on a boundary slot, or INT32_MIN unused
    const int32_t *flags; // bits 0-2: faces of the cell; bit 3+k: cell owns the face of slot k
    // the six per-slot geometry arrays below are consecutive blocks of geoStride values, in this
    // order, starting at aox; geoStride >= n * nSlots is a multiple of 16 bytes so that every
    // component starts 16-byte aligned and 16-byte reads of a block's range stay inside it
    size_t geoStride;
    const T *aox, *aoy, *aoz;        // outward area vector of the slot's face seen from the cell, n A
    const T *dcx, *dcy, *dcz;        // face centre - own cell centre
    const double *vol;               // cell volume
    const double *volP;              // pow(vol, 0.3333) as the reference's CFL bound uses
    // shared-memory staging: blocks of `blockCells` consecutive cells; the face neighbours of a
    // block that lie outside it (its halo) are listed in haloIds[haloStart[b] .. haloStart[b+1]);
    // slotLocal[c * nSlots + k] is the neighbour's index in the block's staged records (own cells
    // first, then the halo), or -bc on a boundary slot.
    int blockCells;
    int maxHalo;
    const int32_t *haloStart;
    const int32_t *haloIds;
    const int16_t *slotLocal;
    // ---- faces (each evaluated once by k_face), in tiles of kFaceTile owner cells: by owner slot,
    //      then owner cell within a tile ----
    int nF;
    size_t fStride;                  // component stride of the face geometry arrays
    const int32_t *fOwn;             // owner cell
    const int32_t *fNb;              // neighbour cell, or -bc on a boundary face
    const T *fnx, *fny, *fnz, *fA;   // canonical unit normal (owner -> neighbour) and area
    const T *fdo[3];                 // face centre - owner centre
    const T *fdn[3];                 // face centre - neighbour centre (periodic image)
    const T *fLsSq;                  // WALE Ls^2 = (0.325 Vavg^0.3333333333333)^2, Vavg = (V_owner +
                                     // V_neighbour) / 2, V_owner on a boundary face
    const int32_t *slotFace;         // [c * nSlots + k] face of a cell slot
    const T *closure;                // [3][n] sum over the cell's faces of outward n * A
};

// face record written by k_face and gathered by k_gather: H[10], u, signal
constexpr int FREC = 12;

// cells per block of the staged stage kernels (FP32 and FP64 records differ in size)
#ifndef FG_STAGE_CELLS_F
#define FG_STAGE_CELLS_F 128
#endif
#ifndef FG_STAGE_CELLS_D
#define FG_STAGE_CELLS_D 64
#endif
// 1: the per-slot geometry of a block is staged in shared memory with its records;
// 0: each face reads its geometry from global memory
#ifndef FG_STAGE_GEOMETRY
#define FG_STAGE_GEOMETRY 0
#endif
// owner cells per tile of the GPU face order (1: by owner cell, then slot).  Tiles of 32 measured
// 1-3 % faster per step than 1 on the 128^3 hex workload (the gather reads nearby records) and
// within 1 % on the graded tet ball.
#ifndef FG_FACE_TILE
#define FG_FACE_TILE 32
#endif
constexpr int kFaceTile = FG_FACE_TILE;
// Minimum resident blocks per SM asked of the compiler (its register budget).  The FP32 stage
// kernels are latency-bound gathers: capping registers at 85 / 85 / 51 per thread (gradient,
// face, gather) raises the warps in flight and measured 2-9 % faster on the 128^3 hex workload.  The
// FP64 gradient and gather kernels need their registers (capping them spills): 0 leaves the choice
// to the compiler.
#ifndef FG_FACE_THREADS
#define FG_FACE_THREADS 64
#endif
#ifndef FG_GATHER_THREADS
#define FG_GATHER_THREADS 128
#endif
#ifndef FG_GRAD_MINB
#define FG_GRAD_MINB 6
#endif
#ifndef FG_FACE_MINB
#define FG_FACE_MINB (6 * 128 / FG_FACE_THREADS)
#endif
#ifndef FG_GATHER_MINB
#define FG_GATHER_MINB (5 * 256 / FG_GATHER_THREADS)
#endif
template <typename T> struct MinBlocks {
    static constexpr int grad = FG_GRAD_MINB, face = FG_FACE_MINB, gather = FG_GATHER_MINB;
};
#ifndef FG_GRAD_MINB_D
#define FG_GRAD_MINB_D 0
#endif
// FP64 face kernel: 6 resident blocks of 64 (168 registers, 88 bytes of spill) measured 15 % faster
// than the compiler's 200 registers (5 blocks) on the 128^3 hex workload
#ifndef FG_FACE_MINB_D
#define FG_FACE_MINB_D 6
#endif
#ifndef FG_GATHER_MINB_D
#define FG_GATHER_MINB_D 0
#endif
template <> struct MinBlocks<double> {
    static constexpr int grad = FG_GRAD_MINB_D, face = FG_FACE_MINB_D, gather = FG_GATHER_MINB_D;
};
template <typename T> struct StageCells { static constexpr int value = FG_STAGE_CELLS_F; };
template <> struct StageCells<double> { static constexpr int value = FG_STAGE_CELLS_D; };

template <typename T>
struct Fields {
    T *FB;              // [nF][FREC] face records
    double *U;          // [10][n]
    double *U0;         // [10][n]
    double *RHS;        // [10][n] (RHS-mode residual)
    T *Win;             // primitive records (WREC values per cell, component-major) read this stage
    T *Wout;            // primitive records written this stage
    T *G;               // limiter + gradient records (GREC values per cell, component-major vectors of
                        // gvec_bytes<T>() bytes, grec_alloc<T>() values per cell allocated)
    double *signal;     // [n]
    T *cellSig;         // [n] per-cell maximum face signal speed of a dt step (zeroed before it)
    double *blockMin;   // [nBlocks]
    double *dt;         // device scalar
    int32_t *bad;       // set to the step counter + 1 when an updated state is not finite or its
                        // mixture density is not positive (sticky until cleared; mapped host memory)
    int32_t step;       // the step counter the kernels record
};

// the updated conserved state of a cell is usable: finite with a positive mixture density (alpha
// itself may leave [0, 1] by rounding: cons2prim clamps it, DP/cons2prim.h:6)
__device__ __forceinline__ bool state_ok(const double *u) {
    double s = 0;
#pragma unroll
    for (int v = 0; v < NV; v++) s += u[v];
    return isfinite(s) && u[1] + u[2] > 0.0;
}

enum FluxMode { FLUX_FUSED = 0, FLUX_RHS = 1 };

struct StageCoef {
    int rk;        // 1 (forward Euler) or 3 (SSP-RK3, Shu-Osher)
    int irk;       // stage
    int writeU0;   // stage 0 of RK3 also stores U0 = U
    int neglectZ;  // the reference's only effective neglect flag (DP/update.cu:26-28)
};

template <typename T>
void launch_grad(const DevMesh<T> &m, const Fields<T> &f, const PhysT<T> &P, cudaStream_t s);
// one-time kernel attribute set-up (dynamic shared memory above 48 KB)
template <typename T>
int stage_kernels_setup(const DevMesh<T> &m);
// wantSignal: 0 none; 1 the face signal speeds into the face records; 2 also their per-cell maxima
// into Fields::cellSig
template <typename T>
void launch_face(const DevMesh<T> &m, const Fields<T> &f, const PhysT<T> &P, int wantSignal, cudaStream_t s);
template <typename T>
void launch_gather(const DevMesh<T> &m, const Fields<T> &f, const PhysD &D, int mode, int wantSignal,
                   StageCoef sc, cudaStream_t s);
template <typename T>
void launch_update(const DevMesh<T> &m, const Fields<T> &f, const PhysD &D, StageCoef sc, cudaStream_t s);
// primitive records of the first n cells from U (records of wStride cells)
template <typename T>
void launch_prim(int n, const double *U, T *W, size_t wStride, const PhysD &D, cudaStream_t s);
// partitioned runs: the records (nval values each, records of nRec cells in vectors of vpv
// values) of cells[0..cnt) to / from a contiguous buffer of whole records
template <typename T>
void launch_halo_pack(const T *rec, size_t nRec, int nval, int vpv, const int32_t *cells, int cnt, T *out,
                      cudaStream_t s);
template <typename T>
void launch_halo_unpack(T *rec, size_t nRec, int nval, int vpv, const int32_t *cells, int cnt, const T *in,
                        cudaStream_t s);
// dt steps of the fused path: per cell (own cells, blocks of the gather kernel) the CFL bound
// volP / cellSig and the signal, the block minima into blockMin[flux_blocks(nU)]
template <typename T>
void launch_cell_cfl(const DevMesh<T> &m, const Fields<T> &f, cudaStream_t s);
// dt = min(cfl * min_blocks, maxDt) from blockMin[nBlocks]
void launch_dt_finalize(const double *blockMin, int nBlocks, double cfl, double maxDt, double *dt, cudaStream_t s);
int flux_blocks(int n);   // blocks of the gather kernel (= entries of blockMin)

// relaxation (FP64 Newton), writes U and the primitive record
struct RelaxParams {
    double gam[2], pinf[2], cp[2], eta[2], satConst[2];
    double avfMin, chemLimit, thermUrf, chemUrf, satTempUrf;
    int thermItrMax, chemItrMax, chemFlag;
};
struct SurrogateDev;
// optional log of chemical Newton solves (training data for the surrogate): X [cap][3], Y [cap][4]
struct RelaxLog {
    float *X;
    float *Y;
    unsigned long long *count;   // null: logging off
    long long cap;
};
// work arrays of the chemical-first cell ordering (n bytes + 4 n + 8 nb + 4 bytes)
struct RelaxOrder {
    uint8_t *isChem;     // [n]
    int32_t *blockCnt;   // [relax_order_blocks(n)]
    int32_t *blockOff;   // [relax_order_blocks(n)]
    int32_t *order;      // [n]
    int32_t *total;      // [1] chemical cells
    float4 *pred;        // [n] surrogate prediction of the chemical cell order[i]
    int32_t *hullOk;     // [n] its input is inside the training hull
    int32_t *tcErr;      // [1] a tensor-core completion wait timed out
    int polishPass;      // with the surrogate: polish in k_relax_polish before the relaxation kernel
};
int relax_order_blocks(int n);
// returns the number of kernels launched
template <typename T>
int launch_relax(int n, double *U, T *W, size_t wStride, const PhysD &D, const RelaxParams &R, int32_t *counters,
                 const SurrogateDev &S, const RelaxLog &L, const RelaxOrder &O, cudaStream_t s);

// conservation integral: blockSum then ordered final sum into out
void launch_cons(int n, int ivar, const double *U, const double *vol, double *blockSum, double *out, cudaStream_t s);
int cons_blocks(int n);
// state probe: out[4] = vapour volume, max / min mixture pressure, max speed (blockOut: 4 per
// cons_blocks(n) block)
void launch_probe(int n, const double *U, const double *vol, const PhysD &D, double *blockOut, double *out,
                  cudaStream_t s);

// first cell of an uploaded AoS state (n x 10) that is not usable, 0x7f7f7f7f if none
void launch_check_state(int n, const double *Uaos, int32_t *firstBad, cudaStream_t s);
// reference-order AoS <-> renumbered SoA
// scatter unless firstBad (set by launch_check_state) names a cell: see k_scatter_state for flags
void launch_scatter_state(int n, const double *Uaos, const int32_t *new2old, double *U, const int32_t *firstBad,
                          int32_t *flags, cudaStream_t s);
void launch_gather_state(int n, const double *U, const int32_t *new2old, double *Uaos, cudaStream_t s);
void launch_copy_u0(int n, const double *U, double *U0, cudaStream_t s);

}  // namespace fg
