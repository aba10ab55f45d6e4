// Space-filling-curve partition of a finished mesh for runs with one GPU per part.
//
// Replaces the reference's METIS decomposition and local-mesh build (DP/decompose.cu:52,
// DP/buildLocalMesh.cu): part p owns the cells of the contiguous range
// [floor(n p / P), floor(n (p+1) / P)) of the mesh's device order (Morton order of the cell
// centres, so a part is a compact region), plus two layers of ghost cells: the first layer, face
// neighbours of own cells in other parts, and the second, their face neighbours in neither.  The
// local mesh keeps every face that touches an own or a first-layer cell with the whole mesh's
// orientation (owner, neighbour), geometry and boundary code, so a part computes the gradients of
// its first-layer ghosts itself, from the same numbers as their owner, and each face flux and each
// cell update from the same numbers as in the unpartitioned run.  Per stage the parts exchange
// only the primitive records of the ghosts (the reference's communicate step, DP/communicate.cu,
// exchanges values and gradients), through the caller's transport.
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
    auto own = [&](int j) { return j >= lo && j < hi; };
    auto dev = [&](int f, int side) { return g.old2new[g.fc2el[2 * f + side]]; };
    // layer 1: the other parts' face neighbours of own cells
    std::vector<uint8_t> layer(n, 0);   // 1 own, 2 first ghost layer, 3 second
    for (int j = lo; j < hi; j++) layer[j] = 1;
    std::vector<int32_t> ghosts1, ghosts2;
    for (int f = 0; f < g.nFcs; f++) {
        if (g.boundCond[f] != 0) continue;
        const int a = dev(f, 0), b = dev(f, 1);
        if (own(a) && !own(b) && !layer[b]) { layer[b] = 2; ghosts1.push_back(b); }
        if (own(b) && !own(a) && !layer[a]) { layer[a] = 2; ghosts1.push_back(a); }
    }
    // layer 2 and the faces: every face touching an own or a first-layer cell
    std::vector<int32_t> faces;
    for (int f = 0; f < g.nFcs; f++) {
        const bool interior = g.boundCond[f] == 0;
        const int a = dev(f, 0), b = interior ? dev(f, 1) : -1;
        const bool inA = layer[a] == 1 || layer[a] == 2, inB = interior && (layer[b] == 1 || layer[b] == 2);
        if (!inA && !inB) continue;
        faces.push_back(f);
        if (interior && !layer[a]) { layer[a] = 3; ghosts2.push_back(a); }
        if (interior && !layer[b]) { layer[b] = 3; ghosts2.push_back(b); }
    }
    std::sort(ghosts1.begin(), ghosts1.end());
    std::sort(ghosts2.begin(), ghosts2.end());
    const int n1 = (int)ghosts1.size();
    const int nL = nOwn + n1 + (int)ghosts2.size();
    // device index of the whole mesh -> local cell: own, then the first layer, then the second
    std::vector<int32_t> localOf(n, -1), globalOf(nL);
    for (int j = lo; j < hi; j++) localOf[j] = j - lo;
    for (int k = 0; k < n1; k++) localOf[ghosts1[k]] = nOwn + k;
    for (size_t k = 0; k < ghosts2.size(); k++) localOf[ghosts2[k]] = nOwn + n1 + (int)k;
    for (int j = 0; j < n; j++)
        if (localOf[j] >= 0) globalOf[localOf[j]] = j;

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
        const int j = globalOf[c];
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
        l.fc2el[2 * i] = localOf[dev(f, 0)];
        l.fc2el[2 * i + 1] = interior ? localOf[dev(f, 1)] : g.fc2el[2 * f + 1];
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
    // halo lists.  A part needs the records of every cell within two face hops of its own cells
    // (its two ghost layers); received grouped by owning part, each group in device order
    std::vector<int32_t> ghostsAll(ghosts1);
    ghostsAll.insert(ghostsAll.end(), ghosts2.begin(), ghosts2.end());
    std::sort(ghostsAll.begin(), ghostsAll.end());
    l.recvStart.assign(P + 1, 0);
    for (int gi : ghostsAll) l.recvStart[part_of(gi) + 1]++;
    for (int q = 0; q < P; q++) l.recvStart[q + 1] += l.recvStart[q];
    l.recvCells.resize(ghostsAll.size());
    for (size_t k = 0; k < ghostsAll.size(); k++) l.recvCells[k] = localOf[ghostsAll[k]];
    // an own cell goes to every other part with a cell within two face hops of it (it is in that
    // part's ghost layers); the local mesh holds every face of its own and first-layer cells
    std::vector<int32_t> adjStart(nL + 1, 0), adj;
    for (int i = 0; i < nF; i++) {
        if (l.boundCond[i] != 0) continue;
        adjStart[l.fc2el[2 * i] + 1]++;
        adjStart[l.fc2el[2 * i + 1] + 1]++;
    }
    for (int c = 0; c < nL; c++) adjStart[c + 1] += adjStart[c];
    adj.resize(adjStart[nL]);
    {
        std::vector<int32_t> fill(adjStart.begin(), adjStart.end() - 1);
        for (int i = 0; i < nF; i++) {
            if (l.boundCond[i] != 0) continue;
            const int a = l.fc2el[2 * i], b = l.fc2el[2 * i + 1];
            adj[fill[a]++] = b;
            adj[fill[b]++] = a;
        }
    }
    std::vector<int64_t> pairs;   // (part, own local cell)
    std::vector<int32_t> seen(P, -1);
    for (int c = 0; c < nOwn; c++) {
        auto mark = [&](int x) {
            const int q = part_of(globalOf[x]);
            if (q != p && seen[q] != c) {
                seen[q] = c;
                pairs.push_back((int64_t)q * nL + c);
            }
        };
        for (int k = adjStart[c]; k < adjStart[c + 1]; k++) {
            const int d = adj[k];
            mark(d);
            for (int k2 = adjStart[d]; k2 < adjStart[d + 1]; k2++) mark(adj[k2]);
        }
    }
    std::sort(pairs.begin(), pairs.end());
    l.sendStart.assign(P + 1, 0);
    l.sendCells.resize(pairs.size());
    for (size_t k = 0; k < pairs.size(); k++) {
        l.sendStart[pairs[k] / nL + 1]++;
        l.sendCells[k] = (int32_t)(pairs[k] % nL);
    }
    for (int q = 0; q < P; q++) l.sendStart[q + 1] += l.sendStart[q];
    l.nOwned = nOwn;
    l.nGhost1 = n1;
    l.nParts = P;
    l.part = p;
    return FG_OK;
}

}  // namespace fg
