// Space-filling-curve partition of a finished mesh for runs with one GPU per part.
//
// Replaces the reference's METIS decomposition and local-mesh build (DP/decompose.cu:52,
// DP/buildLocalMesh.cu): part p owns the cells of the contiguous range
// [floor(n p / P), floor(n (p+1) / P)) of the mesh's device order (Morton order of the cell
// centres, so a part is a compact region), plus one layer of ghost cells, its face neighbours in
// other parts.  The local mesh keeps every face that touches an own cell with the whole mesh's
// orientation (owner, neighbour), geometry and boundary code, so each face flux and each cell
// update is computed from the same numbers as in the unpartitioned run.  Per stage the parts
// exchange the primitive records and then the gradient records of the halo cells (the
// reference's communicate step, DP/communicate.cu), through the caller's transport.
#include "fg_mesh.h"

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

namespace fg {

int partition_mesh(const Mesh &g, int P, int p, Mesh &l, std::string &err) {
    const int n = g.nElem;
    if (g.nOwned >= 0) {
        err = "fg_mesh_partition: the mesh is already a part";
        return FG_ERR_ARG;
    }
    if (P < 1 || p < 0 || p >= P || P > n) {
        err = "fg_mesh_partition: need 1 <= nParts <= cells and 0 <= part < nParts";
        return FG_ERR_ARG;
    }
    auto first = [&](int q) { return (int)((int64_t)n * q / P); };   // first cell (device order) of part q
    auto part_of = [&](int j) {
        int q = (int)((int64_t)j * P / n);
        while (q + 1 < P && first(q + 1) <= j) q++;
        while (q > 0 && first(q) > j) q--;
        return q;
    };
    const int lo = first(p), hi = first(p + 1);
    const int nOwn = hi - lo;
    // faces touching an own cell (whole-mesh face order) and the ghosts they reach
    std::vector<int32_t> faces, ghosts;
    for (int f = 0; f < g.nFcs; f++) {
        const int a = g.old2new[g.fc2el[2 * f]];
        const bool interior = g.boundCond[f] == 0;
        const int b = interior ? g.old2new[g.fc2el[2 * f + 1]] : -1;
        const bool inA = a >= lo && a < hi, inB = interior && b >= lo && b < hi;
        if (!inA && !inB) continue;
        faces.push_back(f);
        if (interior && !inA) ghosts.push_back(a);
        if (interior && !inB) ghosts.push_back(b);
    }
    std::sort(ghosts.begin(), ghosts.end());
    ghosts.erase(std::unique(ghosts.begin(), ghosts.end()), ghosts.end());
    const int nL = nOwn + (int)ghosts.size();
    // device index of the whole mesh -> local cell
    std::vector<int32_t> localOf(n, -1);
    for (int j = lo; j < hi; j++) localOf[j] = j - lo;
    for (size_t k = 0; k < ghosts.size(); k++) localOf[ghosts[k]] = nOwn + (int)k;

    l = Mesh();
    l.nElem = nL;
    l.nNodes = 0;
    l.cellGlobal.resize(nL);
    l.elNN.resize(nL);
    l.elNodes.resize((size_t)nL * 8);
    l.elBc.resize((size_t)nL * 6);
    l.cellCenter.resize((size_t)nL * 3);
    l.elFcCenter.resize((size_t)nL * 18);
    l.volume.resize(nL);
    for (int c = 0; c < nL; c++) {
        const int j = c < nOwn ? lo + c : ghosts[c - nOwn];
        const int e = g.new2old[j];
        l.cellGlobal[c] = e;
        l.elNN[c] = g.elNN[e];
        std::copy_n(&g.elNodes[(size_t)e * 8], 8, &l.elNodes[(size_t)c * 8]);
        std::copy_n(&g.elBc[(size_t)e * 6], 6, &l.elBc[(size_t)c * 6]);
        std::copy_n(&g.cellCenter[(size_t)e * 3], 3, &l.cellCenter[(size_t)c * 3]);
        std::copy_n(&g.elFcCenter[(size_t)e * 18], 18, &l.elFcCenter[(size_t)c * 18]);
        l.volume[c] = g.volume[e];
        switch (l.elNN[c]) {
        case 4: l.nTet++; break;
        case 5: l.nPyr++; break;
        case 6: l.nPrism++; break;
        default: l.nHex++; break;
        }
    }
    const int nF = (int)faces.size();
    l.nFcs = nF;
    l.fc2el.resize((size_t)nF * 2);
    l.fc2elFc.resize((size_t)nF * 2);
    l.boundCond.resize(nF);
    l.fcCenter.resize((size_t)nF * 3);
    l.n.resize((size_t)nF * 3);
    l.nt1.resize((size_t)nF * 3);
    l.nt2.resize((size_t)nF * 3);
    l.area.resize(nF);
    l.nbShift.resize((size_t)nF * 3);
    for (int i = 0; i < nF; i++) {
        const int f = faces[i];
        const bool interior = g.boundCond[f] == 0;
        l.fc2el[2 * i] = localOf[g.old2new[g.fc2el[2 * f]]];
        l.fc2el[2 * i + 1] = interior ? localOf[g.old2new[g.fc2el[2 * f + 1]]] : g.fc2el[2 * f + 1];
        l.fc2elFc[2 * i] = g.fc2elFc[2 * f];
        l.fc2elFc[2 * i + 1] = g.fc2elFc[2 * f + 1];
        l.boundCond[i] = g.boundCond[f];
        l.nBoundary += !interior;
        bool shifted = false;
        for (int d = 0; d < 3; d++) {
            l.fcCenter[(size_t)i * 3 + d] = g.fcCenter[(size_t)f * 3 + d];
            l.n[(size_t)i * 3 + d] = g.n[(size_t)f * 3 + d];
            l.nt1[(size_t)i * 3 + d] = g.nt1[(size_t)f * 3 + d];
            l.nt2[(size_t)i * 3 + d] = g.nt2[(size_t)f * 3 + d];
            l.nbShift[(size_t)i * 3 + d] = g.nbShift[(size_t)f * 3 + d];
            shifted |= g.nbShift[(size_t)f * 3 + d] != 0.0;
        }
        l.nPeriodic += interior && shifted;
        l.area[i] = g.area[f];
    }
    l.maxFaces = g.maxFaces;
    // already in device order: no second renumbering
    l.new2old.resize(nL);
    l.old2new.resize(nL);
    for (int c = 0; c < nL; c++) l.new2old[c] = l.old2new[c] = c;
    // halo lists: ghosts grouped by owning part (ghosts are sorted by device index and the parts
    // are contiguous ranges of it, so the groups are contiguous); own cells sent to each part
    l.recvStart.assign(P + 1, 0);
    for (int gi : ghosts) l.recvStart[part_of(gi) + 1]++;
    for (int q = 0; q < P; q++) l.recvStart[q + 1] += l.recvStart[q];
    l.recvCells.resize(ghosts.size());
    for (size_t k = 0; k < ghosts.size(); k++) l.recvCells[k] = nOwn + (int)k;
    std::vector<int64_t> pairs;   // (part, own local cell)
    for (int i = 0; i < nF; i++) {
        const int a = l.fc2el[2 * i];
        if (l.boundCond[i] != 0) continue;
        const int b = l.fc2el[2 * i + 1];
        if (a < nOwn && b >= nOwn) pairs.push_back((int64_t)part_of(ghosts[b - nOwn]) * nL + a);
        if (b < nOwn && a >= nOwn) pairs.push_back((int64_t)part_of(ghosts[a - nOwn]) * nL + b);
    }
    std::sort(pairs.begin(), pairs.end());
    pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
    l.sendStart.assign(P + 1, 0);
    l.sendCells.resize(pairs.size());
    for (size_t k = 0; k < pairs.size(); k++) {
        l.sendStart[pairs[k] / nL + 1]++;
        l.sendCells[k] = (int32_t)(pairs[k] % nL);
    }
    for (int q = 0; q < P; q++) l.sendStart[q + 1] += l.sendStart[q];
    l.nOwned = nOwn;
    l.nParts = P;
    l.part = p;
    return FG_OK;
}

}  // namespace fg
