// Host-side mesh: Gambit neutral reader, face matching, reference geometry, renumbering.
#pragma once
#include "../../include/fooskagpu.h"

#include <cstdint>
#include <string>
#include <vector>

namespace fg {

// Per-element-type local face tables (Gambit node numbering).
//  kFaceNodesCentre: node order the reference uses to average face centres (DP/translator.cu:146-280)
//  kFaceNodesGeom:   node order the reference uses for normals/areas (DP/operations.h:15-49)
struct ElemType {
    int nNodes;          // 4 tet, 5 pyramid, 6 prism, 8 hex
    int nFaces;
    int faceNodeCount[6];
    int centreNodes[6][4];
    int geomNodes[6][4];
    int volTets;         // tetra split for the volume (DP/meshProperties.cu:168-171)
    int volNodes[6][3];
};
const ElemType *elem_type_for_nodes(int nNodes);

struct Mesh {
    // ---- reference layout (.neu order) ----
    int nElem = 0, nNodes = 0, nFcs = 0;
    std::vector<double> nodes;         // nNodes*3, scaled
    std::vector<int32_t> elNodes;      // nElem*8
    std::vector<int32_t> elNN;         // nodes per element
    std::vector<int32_t> elBc;         // nElem*6 boundary code per local face
    std::vector<double> cellCenter;    // nElem*3
    std::vector<double> elFcCenter;    // nElem*18
    std::vector<int32_t> neig, neigFc; // nElem*6, -1 on boundary
    std::vector<double> neigShift;     // nElem*18 periodic image offset of the neighbour face
    std::vector<int32_t> fc2el, fc2elFc, boundCond;
    std::vector<double> fcCenter, n, nt1, nt2, area, volume, nbShift;
    int nBoundary = 0, nPeriodic = 0, maxFaces = 0;
    int nTet = 0, nPyr = 0, nPrism = 0, nHex = 0;
    // ---- device ordering ----
    std::vector<int32_t> new2old, old2new;
    // ---- part of a partitioned mesh (partition_mesh): cells [0, nOwned) are the part's own,
    // cells [nOwned, nOwned + nGhost1) its first ghost layer (face neighbours owned by other
    // parts: the part computes their gradients, so the mesh holds all their faces), cells
    // [nOwned + nGhost1, nElem) the second layer (their other neighbours: records only) ----
    int nOwned = -1;                       // -1: not partitioned, every cell owned
    int nGhost1 = 0;
    int nParts = 1, part = 0;
    std::vector<int32_t> cellGlobal;       // reference (.neu) index in the whole mesh of each cell
    // cells whose records go to / come from each part q: sendCells[sendStart[q] .. sendStart[q+1])
    // (own cells within two face hops of q's), recvCells[recvStart[q] .. recvStart[q+1]) (ghosts
    // of both layers owned by q), both in the whole mesh's device order, so that the k-th record
    // part p sends to q is q's k-th ghost from p
    std::vector<int32_t> sendStart, sendCells, recvStart, recvCells;
    int owned() const { return nOwned < 0 ? nElem : nOwned; }
    // cells whose gradients the part computes: own and first-layer ghosts
    int gradient_cells() const { return nOwned < 0 ? nElem : nOwned + nGhost1; }
};

// Parse a Gambit neutral file with the reference's grammar (DP/translator.cu:3-354).
// Returns FG_OK or an error code with a message in err.
int read_neu(const std::string &path, double scale, Mesh &m, std::string &err);
// The same element lists handed over in memory: nodes[nNodes*3] (multiplied by scale),
// elNN[nElem], elNodes[nElem*8] (0-based), elBc[nElem*6] (internal codes 0..5).
int mesh_from_arrays(int nNodes, const double *nodes, int nElem, const int32_t *elNN, const int32_t *elNodes,
                     const int32_t *elBc, double scale, Mesh &m, std::string &err);
// Match faces, build the reference face order and geometry, renumber (host).
int finish_mesh(Mesh &m, const fg_mesh_opts &o, std::string &err);
// The same on the GPU (o.device); identical arrays.
int finish_mesh_gpu(Mesh &m, const fg_mesh_opts &o, std::string &err);
// parts shared by both paths
int match_periodic(Mesh &m, const fg_mesh_opts &o, std::vector<int64_t> &unmatched, std::string &err);
int finish_order_geometry(Mesh &m, const fg_mesh_opts &o, std::string &err);
// Part `part` of `nParts` of a finished mesh: the cells of a contiguous range of its device
// (space-filling-curve) order, their ghosts, the faces touching them and the halo lists.
int partition_mesh(const Mesh &g, int nParts, int part, Mesh &l, std::string &err);

}  // namespace fg

struct fg_mesh {
    fg::Mesh m;
};
