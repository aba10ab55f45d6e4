// GPU mesh pre-processor: conforming face matching, the reference face order, face and cell
// geometry and the Morton renumbering on the device, for meshes parsed by read_neu.  Produces
// the same arrays as the host path (finish_mesh) bit for bit: the geometry formulas are the
// same (DP/meshProperties.cu:51-137), evaluated without contracted multiply-adds (this file is
// compiled with --fmad=false) and with x*x for the reference's pow(x, 2), which is the
// correctly rounded square either way.
//
// Matching: every untagged element face gets the key of its sorted node ids (two 64-bit words);
// a stable radix sort by (high, low) brings the two element faces of an interior face next to
// each other.  Faces seen once are open: the host pairs periodic ones (a few percent of the
// faces) as in finish_mesh.  Face order: the element face (e, f) creates a face when it is a
// boundary face or its neighbour has a larger index (DP/buildLocalMesh.cu:263-313); an exclusive
// prefix sum over (e, f) gives the face numbers.
#include "fg_mesh.h"

#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

namespace fg {

namespace {

struct DevTypes {
    int nFaces[9];           // by node count (4 tet, 5 pyramid, 6 prism, 8 hex), 0 otherwise
    int faceNodeCount[9][6];
    int geomNodes[9][6][4];
    int volTets[9];
    int volNodes[9][6][3];
};
__constant__ DevTypes c_types;

template <typename X>
struct DBuf {
    X *p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t k) {
        if (p) cudaFree(p);
        n = k;
        return cudaMalloc(&p, (k ? k : 1) * sizeof(X));
    }
    cudaError_t up(const X *h, size_t k) {
        cudaError_t e = alloc(k);
        if (e != cudaSuccess) return e;
        return cudaMemcpy(p, h, k * sizeof(X), cudaMemcpyHostToDevice);
    }
    cudaError_t down(std::vector<X> &h, size_t k) const {
        h.resize(k);
        return cudaMemcpy(h.data(), p, k * sizeof(X), cudaMemcpyDeviceToHost);
    }
};

constexpr uint64_t kNone = ~0ULL;

// sorted node ids of element face slot s (s = e * 6 + f) as two 64-bit words; kNone for slots
// that are not untagged faces
__global__ void k_keys(int nE, const int32_t *elNN, const int32_t *elNodes, const int32_t *elBc, uint64_t *kHi,
                       uint64_t *kLo, int32_t *slot) {
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= (long long)nE * 6) return;
    const int e = (int)(s / 6), f = (int)(s % 6);
    const int t = elNN[e];
    uint64_t hi = kNone, lo = kNone;
    if (f < c_types.nFaces[t] && elBc[s] == 0) {
        const int cnt = c_types.faceNodeCount[t][f];
        uint32_t v[4] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu};
        for (int i = 0; i < cnt; i++) v[i] = (uint32_t)elNodes[(size_t)e * 8 + c_types.geomNodes[t][f][i]];
        // sort the (up to 4) ids
        for (int i = 1; i < cnt; i++)
            for (int j = i; j > 0 && v[j - 1] > v[j]; j--) {
                const uint32_t x = v[j];
                v[j] = v[j - 1];
                v[j - 1] = x;
            }
        hi = ((uint64_t)v[0] << 32) | v[1];
        lo = ((uint64_t)v[2] << 32) | v[3];
    }
    kHi[s] = hi;
    kLo[s] = lo;
    slot[s] = (int32_t)s;
}

// the high key words in the order of the first sort pass, and the positions 0..n-1
__global__ void k_gather_hi(long long n, const int32_t *slot, const uint64_t *kHi, uint64_t *hiOrd, int32_t *pos) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    hiOrd[i] = kHi[slot[i]];
    pos[i] = (int32_t)i;
}

// final order: low words and slots of the second pass's positions
__global__ void k_permute(long long n, const int32_t *pos, const uint64_t *kLo, const int32_t *slot, uint64_t *loOrd,
                          int32_t *slotOrd) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    loOrd[i] = kLo[pos[i]];
    slotOrd[i] = slot[pos[i]];
}

// pairs of equal adjacent keys become neighbours; single keys are open faces; a key seen more
// than twice (a non-manifold mesh) sets *bad
__global__ void k_match(long long nS, const uint64_t *kHi, const uint64_t *kLo, const int32_t *slot, int32_t *neig,
                        int32_t *neigFc, int32_t *open, int32_t *nOpen, int32_t *bad) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nS || kHi[i] == kNone) return;
    const bool samePrev = i > 0 && kHi[i - 1] == kHi[i] && kLo[i - 1] == kLo[i];
    const bool sameNext = i + 1 < nS && kHi[i + 1] == kHi[i] && kLo[i + 1] == kLo[i];
    if (samePrev && sameNext) {
        *bad = 1;
        return;
    }
    if (sameNext) {
        const int a = slot[i], b = slot[i + 1];
        neig[a] = b / 6;
        neigFc[a] = b % 6;
        neig[b] = a / 6;
        neigFc[b] = a % 6;
    } else if (!samePrev) {
        open[atomicAdd(nOpen, 1)] = slot[i];
    }
}

__global__ void k_creates(int nE, const int32_t *elNN, const int32_t *neig, int32_t *flag) {
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= (long long)nE * 6) return;
    const int e = (int)(s / 6), f = (int)(s % 6);
    const int e1 = neig[s];
    flag[s] = (f < c_types.nFaces[elNN[e]] && (e1 == -1 || e1 > e)) ? 1 : 0;
}

__device__ void normal_vector_d(const double *x, const double *y, const double *z, double *n) {
    const double a = (y[1] - y[0]) * (z[2] - z[0]) - (y[2] - y[0]) * (z[1] - z[0]);
    const double b = (x[1] - x[0]) * (z[2] - z[0]) - (x[2] - x[0]) * (z[1] - z[0]);
    const double c = (x[1] - x[0]) * (y[2] - y[0]) - (x[2] - x[0]) * (y[1] - y[0]);
    const double norm = sqrt(a * a + b * b + c * c);
    n[0] = a / norm;
    n[1] = -b / norm;
    n[2] = c / norm;
}

__device__ void tangent_vectors_d(const double *x, const double *y, const double *z, const double *n, double *t1,
                                  double *t2) {
    const double dx = x[1] - x[0], dy = y[1] - y[0], dz = z[1] - z[0];
    const double norm = sqrt(dx * dx + dy * dy + dz * dz);
    t1[0] = dx / norm;
    t1[1] = dy / norm;
    t1[2] = dz / norm;
    const double a = n[1] * t1[2] - t1[1] * n[2];
    const double b = n[0] * t1[2] - t1[0] * n[2];
    const double c = n[0] * t1[1] - t1[0] * n[1];
    const double norm1 = sqrt(a * a + b * b + c * c);
    t2[0] = a / norm1;
    t2[1] = -b / norm1;
    t2[2] = c / norm1;
}

__device__ double fan_area_d(int nn, const double *x, const double *y, const double *z) {
    double area = 0.0;
    for (int it = 0; it < nn - 2; it++) {
        const double dx1 = x[1 + it] - x[0], dx2 = x[2 + it] - x[0];
        const double dy1 = y[1 + it] - y[0], dy2 = y[2 + it] - y[0];
        const double dz1 = z[1 + it] - z[0], dz2 = z[2 + it] - z[0];
        const double p = dy1 * dz2 - dz1 * dy2, q = dz1 * dx2 - dx1 * dz2, r = dx1 * dy2 - dy1 * dx2;
        area += fabs(0.5 * sqrt(p * p + q * q + r * r));
    }
    return area;
}

struct FaceOut {
    int32_t *fc2el, *fc2elFc, *bc;
    double *fcCenter, *n, *nt1, *nt2, *area, *nbShift;
};

__global__ void k_faces(int nE, const int32_t *elNN, const int32_t *elNodes, const int32_t *elBc, const int32_t *neig,
                        const int32_t *neigFc, const double *neigShift, const double *elFcCenter, const double *nodes,
                        const int32_t *flag, const int32_t *fidx, FaceOut o) {
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= (long long)nE * 6 || !flag[s]) return;
    const int e = (int)(s / 6), lf = (int)(s % 6);
    const int t = elNN[e];
    const int f = fidx[s];
    const int e1 = neig[s];
    o.fc2el[2 * (size_t)f] = e;
    o.fc2el[2 * (size_t)f + 1] = e1;
    o.fc2elFc[2 * (size_t)f] = lf;
    o.fc2elFc[2 * (size_t)f + 1] = (e1 == -1) ? 0 : neigFc[s];
    o.bc[f] = elBc[s];
    double x[4], y[4], z[4];
    const int cnt = c_types.faceNodeCount[t][lf];
    for (int i = 0; i < cnt; i++) {
        const int nd = elNodes[(size_t)e * 8 + c_types.geomNodes[t][lf][i]];
        x[i] = nodes[(size_t)nd * 3 + 0];
        y[i] = nodes[(size_t)nd * 3 + 1];
        z[i] = nodes[(size_t)nd * 3 + 2];
    }
    double nv[3], t1[3], t2[3];
    normal_vector_d(x, y, z, nv);
    tangent_vectors_d(x, y, z, nv, t1, t2);
    for (int d = 0; d < 3; d++) {
        o.n[(size_t)f * 3 + d] = nv[d];
        o.nt1[(size_t)f * 3 + d] = t1[d];
        o.nt2[(size_t)f * 3 + d] = t2[d];
        o.fcCenter[(size_t)f * 3 + d] = elFcCenter[(size_t)e * 18 + lf * 3 + d];
        o.nbShift[(size_t)f * 3 + d] = neigShift[(size_t)s * 3 + d];
    }
    o.area[f] = fan_area_d(cnt, x, y, z);
}

// tetra-split volumes (DP/meshProperties.cu:102-137); *firstBad = smallest element with vol <= 0
__global__ void k_volumes(int nE, const int32_t *elNN, const int32_t *elNodes, const double *nodes, double *volume,
                          int32_t *firstBad) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nE) return;
    const int t = elNN[e];
    const double *p0 = nodes + (size_t)elNodes[(size_t)e * 8 + 0] * 3;
    double vol = 0.0;
    for (int k = 0; k < c_types.volTets[t]; k++) {
        double dx[3], dy[3], dz[3];
        for (int i = 0; i < 3; i++) {
            const double *pi = nodes + (size_t)elNodes[(size_t)e * 8 + c_types.volNodes[t][k][i]] * 3;
            dx[i] = pi[0] - p0[0];
            dy[i] = pi[1] - p0[1];
            dz[i] = pi[2] - p0[2];
        }
        const double c0 = dy[0] * dz[1] - dz[0] * dy[1];
        const double c1 = dz[0] * dx[1] - dx[0] * dz[1];
        const double c2 = dx[0] * dy[1] - dy[0] * dx[1];
        vol += (c0 * dx[2] + c1 * dy[2] + c2 * dz[2]) / 6.0;
    }
    volume[e] = vol;
    if (!(vol > 0.0)) atomicMin(firstBad, e);
}

__device__ uint64_t spread21(uint64_t v) {
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
}

__global__ void k_morton(int nE, const double *cc, double lo0, double lo1, double lo2, double hi0, double hi1,
                         double hi2, uint64_t *key, int32_t *idx) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nE) return;
    const double lo[3] = {lo0, lo1, lo2}, hi[3] = {hi0, hi1, hi2};
    uint32_t q[3];
    for (int d = 0; d < 3; d++) {
        const double span = hi[d] - lo[d];
        const double t = span > 0 ? (cc[(size_t)e * 3 + d] - lo[d]) / span : 0.0;
        q[d] = (uint32_t)fmin(2097151.0, fmax(0.0, t * 2097151.0));
    }
    key[e] = spread21(q[0]) | (spread21(q[1]) << 1) | (spread21(q[2]) << 2);
    idx[e] = e;
}

#define GTRY(expr)                                                                         \
    do {                                                                                   \
        cudaError_t e_ = (expr);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            err = std::string("GPU mesh pre-processor: ") + #expr + ": " + cudaGetErrorString(e_); \
            return e_ == cudaErrorMemoryAllocation ? FG_ERR_NOMEM : FG_ERR_CUDA;           \
        }                                                                                  \
    } while (0)

int upload_types(std::string &err) {
    DevTypes h{};
    for (int nn : {4, 5, 6, 8}) {
        const ElemType *t = elem_type_for_nodes(nn);
        h.nFaces[nn] = t->nFaces;
        h.volTets[nn] = t->volTets;
        for (int f = 0; f < 6; f++) {
            h.faceNodeCount[nn][f] = t->faceNodeCount[f];
            for (int i = 0; i < 4; i++) h.geomNodes[nn][f][i] = t->geomNodes[f][i];
            for (int i = 0; i < 3; i++) h.volNodes[nn][f][i] = t->volNodes[f][i];
        }
    }
    GTRY(cudaMemcpyToSymbol(c_types, &h, sizeof(h)));
    return FG_OK;
}

template <typename K, typename V>
int radix_sort_pairs(DBuf<K> &k, DBuf<V> &v, size_t n, std::string &err) {
    DBuf<K> k2;
    DBuf<V> v2;
    GTRY(k2.alloc(n));
    GTRY(v2.alloc(n));
    size_t tmp = 0;
    GTRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp, k.p, k2.p, v.p, v2.p, (int64_t)n));
    DBuf<unsigned char> t;
    GTRY(t.alloc(tmp));
    GTRY(cub::DeviceRadixSort::SortPairs(t.p, tmp, k.p, k2.p, v.p, v2.p, (int64_t)n));
    std::swap(k.p, k2.p);
    std::swap(v.p, v2.p);
    return FG_OK;
}

}  // namespace

// periodic matching of the open faces (host, shared with finish_mesh)
int match_periodic(Mesh &m, const fg_mesh_opts &o, std::vector<int64_t> &unmatched, std::string &err);

int finish_mesh_gpu(Mesh &m, const fg_mesh_opts &o, std::string &err) {
    const int nE = m.nElem;
    const size_t nS = (size_t)nE * 6;
    GTRY(cudaSetDevice(o.device));
    int rc = upload_types(err);
    if (rc != FG_OK) return rc;
    DBuf<int32_t> dNN, dElNodes, dBc, dNeig, dNeigFc, dOpen, dCnt;
    GTRY(dNN.up(m.elNN.data(), nE));
    GTRY(dElNodes.up(m.elNodes.data(), (size_t)nE * 8));
    GTRY(dBc.up(m.elBc.data(), nS));
    GTRY(dNeig.alloc(nS));
    GTRY(dNeigFc.alloc(nS));
    GTRY(cudaMemset(dNeig.p, 0xff, nS * sizeof(int32_t)));   // -1
    GTRY(cudaMemset(dNeigFc.p, 0, nS * sizeof(int32_t)));
    GTRY(dOpen.alloc(nS));
    GTRY(dCnt.alloc(2));
    GTRY(cudaMemset(dCnt.p, 0, 2 * sizeof(int32_t)));
    const int T = 256;
    const unsigned gS = (unsigned)((nS + T - 1) / T);
    // ---- conforming matching
    {
        DBuf<uint64_t> kHi, kLo, hiOrd;
        DBuf<int32_t> slot, pos, slotOrd;
        GTRY(kHi.alloc(nS));
        GTRY(kLo.alloc(nS));
        GTRY(slot.alloc(nS));
        k_keys<<<gS, T>>>(nE, dNN.p, dElNodes.p, dBc.p, kHi.p, kLo.p, slot.p);
        GTRY(cudaGetLastError());
        // lexicographic (hi, lo) order by two stable passes: by lo, then by hi
        rc = radix_sort_pairs(kLo, slot, nS, err);       // kLo, slot in lo order
        if (rc != FG_OK) return rc;
        GTRY(hiOrd.alloc(nS));
        GTRY(pos.alloc(nS));
        k_gather_hi<<<gS, T>>>((long long)nS, slot.p, kHi.p, hiOrd.p, pos.p);
        GTRY(cudaGetLastError());
        rc = radix_sort_pairs(hiOrd, pos, nS, err);      // hiOrd sorted, pos = index into lo order
        if (rc != FG_OK) return rc;
        DBuf<uint64_t> loOrd;
        GTRY(loOrd.alloc(nS));
        GTRY(slotOrd.alloc(nS));
        k_permute<<<gS, T>>>((long long)nS, pos.p, kLo.p, slot.p, loOrd.p, slotOrd.p);
        GTRY(cudaGetLastError());
        k_match<<<gS, T>>>((long long)nS, hiOrd.p, loOrd.p, slotOrd.p, dNeig.p, dNeigFc.p, dOpen.p, dCnt.p,
                           dCnt.p + 1);
        GTRY(cudaGetLastError());
    }
    int32_t cnt[2];
    GTRY(cudaMemcpy(cnt, dCnt.p, sizeof(cnt), cudaMemcpyDeviceToHost));
    if (cnt[1]) {
        err = "non-manifold mesh: a face is shared by more than two elements";
        return FG_ERR_MESH;
    }
    GTRY(dNeig.down(m.neig, nS));
    GTRY(dNeigFc.down(m.neigFc, nS));
    std::vector<int32_t> op;
    GTRY(dOpen.down(op, (size_t)cnt[0]));
    std::vector<int64_t> unmatched(op.begin(), op.end());
    std::sort(unmatched.begin(), unmatched.end());
    m.neigShift.assign(nS * 3, 0.0);
    rc = match_periodic(m, o, unmatched, err);
    if (rc != FG_OK) return rc;
    // ---- the reference face order, face geometry, volumes
    GTRY(dNeig.up(m.neig.data(), nS));
    GTRY(dNeigFc.up(m.neigFc.data(), nS));
    DBuf<double> dShift, dElFc, dNodes;
    GTRY(dShift.up(m.neigShift.data(), nS * 3));
    GTRY(dElFc.up(m.elFcCenter.data(), nS * 3));
    GTRY(dNodes.up(m.nodes.data(), (size_t)m.nNodes * 3));
    DBuf<int32_t> flag, fidx;
    GTRY(flag.alloc(nS));
    GTRY(fidx.alloc(nS));
    k_creates<<<gS, T>>>(nE, dNN.p, dNeig.p, flag.p);
    GTRY(cudaGetLastError());
    {
        size_t tmp = 0;
        GTRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp, flag.p, fidx.p, (int64_t)nS));
        DBuf<unsigned char> t;
        GTRY(t.alloc(tmp));
        GTRY(cub::DeviceScan::ExclusiveSum(t.p, tmp, flag.p, fidx.p, (int64_t)nS));
    }
    int32_t lastIdx = 0, lastFlag = 0;
    GTRY(cudaMemcpy(&lastIdx, fidx.p + nS - 1, sizeof(int32_t), cudaMemcpyDeviceToHost));
    GTRY(cudaMemcpy(&lastFlag, flag.p + nS - 1, sizeof(int32_t), cudaMemcpyDeviceToHost));
    const int nF = lastIdx + lastFlag;
    DBuf<int32_t> fc2el, fc2elFc, bc;
    DBuf<double> fcC, fn, ft1, ft2, farea, fsh, vol;
    GTRY(fc2el.alloc((size_t)nF * 2));
    GTRY(fc2elFc.alloc((size_t)nF * 2));
    GTRY(bc.alloc(nF));
    for (DBuf<double> *b : {&fcC, &fn, &ft1, &ft2, &fsh}) GTRY(b->alloc((size_t)nF * 3));
    GTRY(farea.alloc(nF));
    GTRY(vol.alloc(nE));
    FaceOut fo{fc2el.p, fc2elFc.p, bc.p, fcC.p, fn.p, ft1.p, ft2.p, farea.p, fsh.p};
    k_faces<<<gS, T>>>(nE, dNN.p, dElNodes.p, dBc.p, dNeig.p, dNeigFc.p, dShift.p, dElFc.p, dNodes.p, flag.p, fidx.p,
                       fo);
    GTRY(cudaGetLastError());
    GTRY(cudaMemcpy(dCnt.p, &nE, sizeof(int32_t), cudaMemcpyHostToDevice));   // first bad element
    k_volumes<<<(nE + T - 1) / T, T>>>(nE, dNN.p, dElNodes.p, dNodes.p, vol.p, dCnt.p);
    GTRY(cudaGetLastError());
    int32_t firstBad = nE;
    GTRY(cudaMemcpy(&firstBad, dCnt.p, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (firstBad < nE) {
        err = "element " + std::to_string(firstBad + 1) + " has non-positive volume (inverted node order)";
        return FG_ERR_MESH;
    }
    m.nFcs = nF;
    GTRY(fc2el.down(m.fc2el, (size_t)nF * 2));
    GTRY(fc2elFc.down(m.fc2elFc, (size_t)nF * 2));
    GTRY(bc.down(m.boundCond, nF));
    GTRY(fcC.down(m.fcCenter, (size_t)nF * 3));
    GTRY(fn.down(m.n, (size_t)nF * 3));
    GTRY(ft1.down(m.nt1, (size_t)nF * 3));
    GTRY(ft2.down(m.nt2, (size_t)nF * 3));
    GTRY(fsh.down(m.nbShift, (size_t)nF * 3));
    GTRY(farea.down(m.area, nF));
    GTRY(vol.down(m.volume, nE));
    m.maxFaces = 0;
    for (int e = 0; e < nE; e++) m.maxFaces = std::max(m.maxFaces, elem_type_for_nodes(m.elNN[e])->nFaces);
    m.nBoundary = 0;
    for (int f = 0; f < nF; f++) m.nBoundary += (m.boundCond[f] != 0);
    // ---- device ordering
    m.new2old.resize(nE);
    if (o.renumber == FG_RENUMBER_MORTON) {
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int e = 0; e < nE; e++)
            for (int d = 0; d < 3; d++) {
                lo[d] = std::min(lo[d], m.cellCenter[(size_t)e * 3 + d]);
                hi[d] = std::max(hi[d], m.cellCenter[(size_t)e * 3 + d]);
            }
        DBuf<double> dcc;
        DBuf<uint64_t> key;
        DBuf<int32_t> idx;
        GTRY(dcc.up(m.cellCenter.data(), (size_t)nE * 3));
        GTRY(key.alloc(nE));
        GTRY(idx.alloc(nE));
        k_morton<<<(nE + T - 1) / T, T>>>(nE, dcc.p, lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], key.p, idx.p);
        GTRY(cudaGetLastError());
        rc = radix_sort_pairs(key, idx, nE, err);   // stable: equal keys keep the element order
        if (rc != FG_OK) return rc;
        GTRY(idx.down(m.new2old, nE));
    } else if (o.renumber == FG_RENUMBER_RCM) {
        err = "the GPU pre-processor renumbers along the Morton curve only (use the host path for RCM)";
        return FG_ERR_UNSUPPORTED;
    } else {
        std::iota(m.new2old.begin(), m.new2old.end(), 0);
    }
    m.old2new.resize(nE);
    for (int i = 0; i < nE; i++) m.old2new[m.new2old[i]] = i;
    return FG_OK;
}

}  // namespace fg
