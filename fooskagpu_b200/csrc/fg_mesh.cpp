// Host mesh pre-processing for the device path.
//
// Reference behaviour restated here (single rank):
//   - Gambit neutral grammar and section detection: DP/translator.cu:24-349
//   - cell centres and per-element face centres: DP/translator.cu:122-282
//   - face matching (the reference compares face centres among elements sharing a node,
//     DP/meshConnectivity.cu:97-128; conforming meshes give the same pairs as matching the
//     sorted node sets, which is what is done here)
//   - face order and ownership (owner = first element in file order, faces in element /
//     local-face order): DP/buildLocalMesh.cu:263-313 with one partition
//   - normals, tangents, areas, volumes: DP/meshProperties.cu:51-180
// Extensions: periodic matching of untagged boundary faces, Morton / RCM renumbering.
#include "fg_mesh.h"

#include <algorithm>
#include <array>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <queue>
#include <unordered_map>

namespace fg {

static const ElemType kTet = {
    4, 4, {3, 3, 3, 3, 0, 0},
    {{1, 0, 2, -1}, {0, 1, 3, -1}, {1, 2, 3, -1}, {2, 0, 3, -1}, {-1, -1, -1, -1}, {-1, -1, -1, -1}},
    {{1, 0, 2, -1}, {0, 1, 3, -1}, {1, 2, 3, -1}, {2, 0, 3, -1}, {-1, -1, -1, -1}, {-1, -1, -1, -1}},
    1, {{1, 2, 3}}};
static const ElemType kPyr = {
    5, 5, {4, 3, 3, 3, 3, 0},
    {{0, 2, 3, 1}, {0, 1, 4, -1}, {1, 3, 4, -1}, {3, 2, 4, -1}, {2, 0, 4, -1}, {-1, -1, -1, -1}},
    {{0, 2, 3, 1}, {0, 1, 4, -1}, {1, 3, 4, -1}, {3, 2, 4, -1}, {2, 0, 4, -1}, {-1, -1, -1, -1}},
    2, {{1, 3, 4}, {3, 2, 4}}};
static const ElemType kPrism = {
    6, 5, {4, 4, 4, 3, 3, 0},
    {{0, 1, 4, 3}, {1, 2, 5, 4}, {2, 0, 3, 5}, {0, 2, 1, -1}, {3, 4, 5, -1}, {-1, -1, -1, -1}},
    {{0, 1, 4, 3}, {2, 5, 4, 1}, {0, 3, 5, 2}, {0, 2, 1, -1}, {3, 4, 5, -1}, {-1, -1, -1, -1}},
    3, {{1, 2, 5}, {1, 5, 4}, {4, 5, 3}}};
static const ElemType kHex = {
    8, 6, {4, 4, 4, 4, 4, 4},
    {{0, 1, 5, 4}, {1, 3, 7, 5}, {3, 2, 6, 7}, {2, 0, 4, 6}, {1, 0, 2, 3}, {4, 5, 7, 6}},
    {{0, 1, 5, 4}, {3, 7, 5, 1}, {2, 6, 7, 3}, {2, 0, 4, 6}, {2, 3, 1, 0}, {6, 4, 5, 7}},
    6, {{1, 3, 5}, {5, 3, 7}, {5, 7, 4}, {3, 2, 7}, {7, 2, 6}, {7, 6, 4}}};

const ElemType *elem_type_for_nodes(int nn) {
    switch (nn) {
    case 4: return &kTet;
    case 5: return &kPyr;
    case 6: return &kPrism;
    case 8: return &kHex;
    default: return nullptr;
    }
}

// ------------------------------------------------------------------ .neu reader
namespace {

struct Reader {
    const char *p, *end;
    int line = 1;
    bool eof() const { return p >= end; }
    // read one line into s (without newline); returns false at EOF
    bool getline(std::string &s) {
        if (p >= end) return false;
        const char *q = p;
        while (q < end && *q != '\n') q++;
        s.assign(p, q);
        if (!s.empty() && s.back() == '\r') s.pop_back();
        p = (q < end) ? q + 1 : q;
        line++;
        return true;
    }
    void skipws() {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) {
            if (*p == '\n') line++;
            p++;
        }
    }
    bool get_long(long &v) {
        skipws();
        if (p >= end) return false;
        char *e;
        errno = 0;
        v = strtol(p, &e, 10);
        if (e == p || errno) return false;
        p = e;
        return true;
    }
    bool get_double(double &v) {
        skipws();
        if (p >= end) return false;
        char *e;
        v = strtod(p, &e);
        if (e == p) return false;
        p = e;
        return true;
    }
    bool get_word(std::string &w) {
        skipws();
        if (p >= end) return false;
        const char *q = p;
        while (q < end && !(*q == ' ' || *q == '\t' || *q == '\r' || *q == '\n')) q++;
        w.assign(p, q);
        p = q;
        return true;
    }
    // advance to the line whose first 20 characters equal the 20-character prefix of key
    bool seek_section(const char *key) {
        std::string s;
        while (getline(s)) {
            if (s.size() >= 20 ? s.compare(0, 20, key, 20) == 0 : false) return true;
        }
        return false;
    }
};

// 20-character section prefixes as compared by the reference (strncmp(..., 20))
const char kCtrl[] = "CONTROL INFO        ";
const char kNodes[] = "NODAL COORDINATES   ";
const char kElems[] = "ELEMENTS/CELLS      ";
const char kBcs[] = "BOUNDARY CONDITIONS ";

}  // namespace

// Cell centres, per-element face centres and element-type counts from the element lists.
static void finish_elements(Mesh &m) {
    const size_t elnum = (size_t)m.nElem;
    m.cellCenter.assign(elnum * 3, 0.0);
    m.elFcCenter.assign(elnum * 18, 0.0);
    m.nTet = m.nPyr = m.nPrism = m.nHex = 0;
    for (size_t e = 0; e < elnum; e++) {
        const int nc = m.elNN[e];
        const ElemType *et = elem_type_for_nodes(nc);
        // cell centre: plain average in node order (DP/translator.cu:138-143, 183-188, 223-228, 261-263)
        for (int d = 0; d < 3; d++) {
            double sum = m.nodes[(size_t)m.elNodes[e * 8 + 0] * 3 + d];
            for (int k = 1; k < nc; k++) sum = sum + m.nodes[(size_t)m.elNodes[e * 8 + k] * 3 + d];
            m.cellCenter[e * 3 + d] = sum / nc;
        }
        // face centres in the reference's node order
        for (int f = 0; f < et->nFaces; f++) {
            const int cnt = et->faceNodeCount[f];
            for (int d = 0; d < 3; d++) {
                double sum = m.nodes[(size_t)m.elNodes[e * 8 + et->centreNodes[f][0]] * 3 + d];
                for (int k = 1; k < cnt; k++) sum = sum + m.nodes[(size_t)m.elNodes[e * 8 + et->centreNodes[f][k]] * 3 + d];
                m.elFcCenter[e * 18 + f * 3 + d] = sum / cnt;
            }
        }
        switch (nc) {
        case 4: m.nTet++; break;
        case 5: m.nPyr++; break;
        case 6: m.nPrism++; break;
        default: m.nHex++; break;
        }
    }
}

int read_neu(const std::string &path, double scale, Mesh &m, std::string &err) {
    FILE *fp = fopen(path.c_str(), "rb");
    if (!fp) {
        err = "mesh file not found: " + path;
        return FG_ERR_IO;
    }
    std::vector<char> buf;
    {
        fseek(fp, 0, SEEK_END);
        long sz = ftell(fp);
        fseek(fp, 0, SEEK_SET);
        if (sz < 0) { fclose(fp); err = "cannot size mesh file"; return FG_ERR_IO; }
        buf.resize((size_t)sz);
        if (sz > 0 && fread(buf.data(), 1, (size_t)sz, fp) != (size_t)sz) {
            fclose(fp);
            err = "short read on mesh file";
            return FG_ERR_IO;
        }
        fclose(fp);
    }
    Reader r{buf.data(), buf.data() + buf.size()};
    std::string s;
    if (!r.seek_section(kCtrl)) { err = "no CONTROL INFO section"; return FG_ERR_MESH; }
    for (int i = 0; i < 5; i++)
        if (!r.getline(s)) { err = "truncated CONTROL INFO"; return FG_ERR_MESH; }
    long ndnum, elnum, code1, bcnum, dim, code2;
    if (!r.get_long(ndnum) || !r.get_long(elnum) || !r.get_long(code1) || !r.get_long(bcnum) ||
        !r.get_long(dim) || !r.get_long(code2)) {
        err = "bad CONTROL INFO counts";
        return FG_ERR_MESH;
    }
    if (ndnum <= 0 || elnum <= 0 || bcnum < 0 || ndnum > (1L << 30) || elnum > (1L << 28)) {
        err = "CONTROL INFO counts out of range";
        return FG_ERR_MESH;
    }
    (void)code1; (void)dim; (void)code2;
    if (!r.seek_section(kNodes)) { err = "no NODAL COORDINATES section"; return FG_ERR_MESH; }
    m.nNodes = (int)ndnum;
    m.nElem = (int)elnum;
    m.nodes.resize((size_t)ndnum * 3);
    for (long i = 0; i < ndnum; i++) {
        long id;
        double x, y, z;
        if (!r.get_long(id) || !r.get_double(x) || !r.get_double(y) || !r.get_double(z)) {
            err = "truncated node list at node " + std::to_string(i + 1);
            return FG_ERR_MESH;
        }
        m.nodes[i * 3 + 0] = x * scale;
        m.nodes[i * 3 + 1] = y * scale;
        m.nodes[i * 3 + 2] = z * scale;
    }
    if (!r.seek_section(kElems)) { err = "no ELEMENTS/CELLS section"; return FG_ERR_MESH; }
    m.elNodes.assign((size_t)elnum * 8, 0);
    m.elNN.assign(elnum, 0);
    m.elBc.assign((size_t)elnum * 6, 0);
    std::vector<char> seen(elnum, 0);
    for (long i = 0; i < elnum; i++) {
        long el, typ, nc;
        if (!r.get_long(el) || !r.get_long(typ) || !r.get_long(nc)) {
            err = "truncated element list at entry " + std::to_string(i + 1);
            return FG_ERR_MESH;
        }
        const ElemType *et = elem_type_for_nodes((int)nc);
        if (!et) { err = "unsupported element with " + std::to_string(nc) + " nodes"; return FG_ERR_MESH; }
        if (el < 1 || el > elnum || seen[el - 1]) { err = "bad or repeated element id " + std::to_string(el); return FG_ERR_MESH; }
        seen[el - 1] = 1;
        const long e = el - 1;
        for (int k = 0; k < nc; k++) {
            long c;
            if (!r.get_long(c)) { err = "truncated element connectivity"; return FG_ERR_MESH; }
            if (c < 1 || c > ndnum) { err = "node id out of range in element " + std::to_string(el); return FG_ERR_MESH; }
            m.elNodes[e * 8 + k] = (int32_t)(c - 1);
        }
        m.elNN[e] = (int32_t)nc;
    }
    if (!r.seek_section(kBcs)) {
        if (bcnum > 0) { err = "no BOUNDARY CONDITIONS section"; return FG_ERR_MESH; }
        finish_elements(m);
        return FG_OK;
    }
    for (long b = 0; b < bcnum; b++) {
        std::string name;
        long und1, nent, und2, code;
        if (!r.get_word(name) || !r.get_long(und1) || !r.get_long(nent) || !r.get_long(und2) || !r.get_long(code)) {
            err = "bad boundary condition header";
            return FG_ERR_MESH;
        }
        // IBCCODE -> internal code (DP/translator.cu:304-343)
        int bc = 0;
        if (code == 45) bc = 1;        // symmetry
        else if (code == 26) bc = 2;   // outlet
        else if (code == 13) bc = 3;   // inlet
        else if (code == 42) bc = 4;   // slip wall
        else if (code == 51) bc = 5;   // wall
        for (long i = 0; i < nent; i++) {
            long el, typ, face;
            if (!r.get_long(el) || !r.get_long(typ) || !r.get_long(face)) { err = "truncated boundary entries"; return FG_ERR_MESH; }
            if (el < 1 || el > elnum || face < 1 || face > 6) { err = "boundary entry out of range"; return FG_ERR_MESH; }
            if (bc != 0) m.elBc[(el - 1) * 6 + (face - 1)] = bc;  // unknown codes leave the face untagged
        }
        if (b != bcnum - 1) {
            // ENDOFSECTION and the next section header
            r.skipws();
            if (!r.getline(s) || !r.getline(s)) { err = "truncated boundary sections"; return FG_ERR_MESH; }
        }
    }
    for (long e = 0; e < elnum; e++)
        if (!seen[e]) { err = "element " + std::to_string(e + 1) + " missing"; return FG_ERR_MESH; }
    finish_elements(m);
    return FG_OK;
}

int mesh_from_arrays(int nNodes, const double *nodes, int nElem, const int32_t *elNN, const int32_t *elNodes,
                     const int32_t *elBc, double scale, Mesh &m, std::string &err) {
    if (nNodes <= 0 || nElem <= 0 || nElem > (1 << 28)) { err = "node / element counts out of range"; return FG_ERR_ARG; }
    m.nNodes = nNodes;
    m.nElem = nElem;
    m.nodes.resize((size_t)nNodes * 3);
    for (size_t i = 0; i < (size_t)nNodes * 3; i++) m.nodes[i] = nodes[i] * scale;
    m.elNodes.assign((size_t)nElem * 8, 0);
    m.elNN.assign(nElem, 0);
    m.elBc.assign((size_t)nElem * 6, 0);
    for (size_t e = 0; e < (size_t)nElem; e++) {
        const int nc = elNN[e];
        const ElemType *et = elem_type_for_nodes(nc);
        if (!et) { err = "unsupported element with " + std::to_string(nc) + " nodes at " + std::to_string(e); return FG_ERR_MESH; }
        m.elNN[e] = nc;
        for (int k = 0; k < nc; k++) {
            const int32_t c = elNodes[e * 8 + k];
            if (c < 0 || c >= nNodes) { err = "node id out of range in element " + std::to_string(e); return FG_ERR_MESH; }
            m.elNodes[e * 8 + k] = c;
        }
        for (int f = 0; f < 6; f++) {
            const int32_t bc = elBc[e * 6 + f];
            if (bc < 0 || bc > 5 || (bc != 0 && f >= et->nFaces)) {
                err = "boundary code out of range at element " + std::to_string(e) + " face " + std::to_string(f);
                return FG_ERR_MESH;
            }
            m.elBc[e * 6 + f] = bc;
        }
    }
    finish_elements(m);
    return FG_OK;
}

// ------------------------------------------------------------------ geometry (DP/meshProperties.cu:51-137)
static void normal_vector(const double *x, const double *y, const double *z, double *n) {
    const double a = (y[1] - y[0]) * (z[2] - z[0]) - (y[2] - y[0]) * (z[1] - z[0]);
    const double b = (x[1] - x[0]) * (z[2] - z[0]) - (x[2] - x[0]) * (z[1] - z[0]);
    const double c = (x[1] - x[0]) * (y[2] - y[0]) - (x[2] - x[0]) * (y[1] - y[0]);
    const double norm = sqrt(pow(a, 2.0) + pow(b, 2.0) + pow(c, 2.0));
    n[0] = a / norm;
    n[1] = -b / norm;
    n[2] = c / norm;
}

static void tangent_vectors(const double *x, const double *y, const double *z, const double *n, double *t1, double *t2) {
    const double norm = sqrt(pow(x[1] - x[0], 2.0) + pow(y[1] - y[0], 2.0) + pow(z[1] - z[0], 2.0));
    t1[0] = (x[1] - x[0]) / norm;
    t1[1] = (y[1] - y[0]) / norm;
    t1[2] = (z[1] - z[0]) / norm;
    const double a = n[1] * t1[2] - t1[1] * n[2];
    const double b = n[0] * t1[2] - t1[0] * n[2];
    const double c = n[0] * t1[1] - t1[0] * n[1];
    const double norm1 = sqrt(pow(a, 2.0) + pow(b, 2.0) + pow(c, 2.0));
    t2[0] = a / norm1;
    t2[1] = -b / norm1;
    t2[2] = c / norm1;
}

static double fan_area(int nn, const double *x, const double *y, const double *z) {
    double area = 0.0;
    for (int it = 0; it < nn - 2; it++) {
        const double dx1 = x[1 + it] - x[0], dx2 = x[2 + it] - x[0];
        const double dy1 = y[1 + it] - y[0], dy2 = y[2 + it] - y[0];
        const double dz1 = z[1 + it] - z[0], dz2 = z[2 + it] - z[0];
        area += fabs(0.5 * sqrt(pow(dy1 * dz2 - dz1 * dy2, 2) + pow(dz1 * dx2 - dx1 * dz2, 2) + pow(dx1 * dy2 - dy1 * dx2, 2)));
    }
    return area;
}

// ------------------------------------------------------------------ face matching
namespace {
struct FaceKey {
    std::array<int32_t, 4> v;
    bool operator==(const FaceKey &o) const { return v == o.v; }
};
struct FaceKeyHash {
    size_t operator()(const FaceKey &k) const {
        uint64_t h = 1469598103934665603ULL;
        for (int i = 0; i < 4; i++) {
            h ^= (uint64_t)(uint32_t)k.v[i];
            h *= 1099511628211ULL;
        }
        return (size_t)h;
    }
};

uint64_t morton3(uint32_t x, uint32_t y, uint32_t z) {
    auto spread = [](uint64_t v) {
        v &= 0x1fffff;
        v = (v | v << 32) & 0x1f00000000ffffULL;
        v = (v | v << 16) & 0x1f0000ff0000ffULL;
        v = (v | v << 8) & 0x100f00f00f00f00fULL;
        v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
        v = (v | v << 2) & 0x1249249249249249ULL;
        return v;
    };
    return spread(x) | (spread(y) << 1) | (spread(z) << 2);
}
}  // namespace

int finish_mesh(Mesh &m, const fg_mesh_opts &o, std::string &err) {
    const int nE = m.nElem;
    m.neig.assign((size_t)nE * 6, -1);
    m.neigFc.assign((size_t)nE * 6, 0);
    m.neigShift.assign((size_t)nE * 18, 0.0);
    // conforming matching on sorted node sets of untagged faces
    std::unordered_map<FaceKey, int64_t, FaceKeyHash> open;
    open.reserve((size_t)nE * 3);
    std::vector<int64_t> unmatched;
    for (int e = 0; e < nE; e++) {
        const ElemType *et = elem_type_for_nodes(m.elNN[e]);
        for (int f = 0; f < et->nFaces; f++) {
            if (m.elBc[(size_t)e * 6 + f] != 0) continue;
            FaceKey k;
            k.v = {-1, -1, -1, -1};
            const int cnt = et->faceNodeCount[f];
            for (int i = 0; i < cnt; i++) k.v[i] = m.elNodes[(size_t)e * 8 + et->geomNodes[f][i]];
            std::sort(k.v.begin(), k.v.begin() + cnt);
            auto it = open.find(k);
            if (it == open.end()) {
                open.emplace(k, (int64_t)e * 6 + f);
            } else {
                const int64_t other = it->second;
                const int e1 = (int)(other / 6), f1 = (int)(other % 6);
                m.neig[(size_t)e * 6 + f] = e1;
                m.neigFc[(size_t)e * 6 + f] = f1;
                m.neig[(size_t)e1 * 6 + f1] = e;
                m.neigFc[(size_t)e1 * 6 + f1] = f;
                open.erase(it);
            }
        }
    }
    for (auto &kv : open) unmatched.push_back(kv.second);
    std::sort(unmatched.begin(), unmatched.end());
    const int rc = match_periodic(m, o, unmatched, err);
    if (rc != FG_OK) return rc;
    return finish_order_geometry(m, o, err);
}

// Pair the open (unmatched, untagged) element faces periodically when the options ask for it;
// any face still open is an error.  unmatched is sorted.
int match_periodic(Mesh &m, const fg_mesh_opts &o, std::vector<int64_t> &unmatched, std::string &err) {
    m.nPeriodic = 0;
    // periodic matching (extension): pair untagged open faces whose centres differ by a box length
    const bool anyPer = o.periodic[0] > 0 || o.periodic[1] > 0 || o.periodic[2] > 0;
    if (!unmatched.empty() && anyPer) {
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int i = 0; i < m.nNodes; i++)
            for (int d = 0; d < 3; d++) {
                lo[d] = std::min(lo[d], m.nodes[(size_t)i * 3 + d]);
                hi[d] = std::max(hi[d], m.nodes[(size_t)i * 3 + d]);
            }
        double L[3];
        for (int d = 0; d < 3; d++) L[d] = o.periodic[d] * o.scale;
        double span = 0;
        for (int d = 0; d < 3; d++) span = std::max(span, hi[d] - lo[d]);
        const double tol = 1e-7 * (span > 0 ? span : 1.0);
        // face centre wrapped into the periodic box; faces whose wrapped centres are within tol
        // (per axis, modulo L) are periodic images of each other
        auto wrap = [&](const double *c, double *w) {
            for (int d = 0; d < 3; d++) {
                double v = c[d];
                if (L[d] > 0) {
                    v = v - lo[d];
                    v = v - L[d] * std::floor(v / L[d] + 0.5 * tol / L[d]);
                    if (v > L[d] - tol) v -= L[d];
                }
                w[d] = v;
            }
        };
        // hash grid of cell size 4 tol: an image lies in the same or an adjacent cell
        auto cellOf = [&](const double *w) {
            std::array<int64_t, 3> k;
            for (int d = 0; d < 3; d++) k[d] = (int64_t)std::floor(w[d] / (4 * tol));
            return k;
        };
        struct AH {
            size_t operator()(const std::array<int64_t, 3> &a) const {
                return (size_t)(a[0] * 73856093LL ^ a[1] * 19349663LL ^ a[2] * 83492791LL);
            }
        };
        const size_t nU = unmatched.size();
        std::vector<double> wc(nU * 3);
        std::unordered_map<std::array<int64_t, 3>, std::vector<int64_t>, AH> grid;
        grid.reserve(nU);
        for (size_t i = 0; i < nU; i++) {
            wrap(&m.elFcCenter[(size_t)unmatched[i] * 3], &wc[i * 3]);
            grid[cellOf(&wc[i * 3])].push_back((int64_t)i);
        }
        std::vector<char> done(nU, 0);
        auto near = [&](size_t i, size_t j) {
            for (int d = 0; d < 3; d++) {
                double dd = std::fabs(wc[i * 3 + d] - wc[j * 3 + d]);
                if (L[d] > 0) dd = std::min(dd, std::fabs(L[d] - dd));
                if (dd > tol) return false;
            }
            return true;
        };
        for (size_t i = 0; i < nU; i++) {
            if (done[i]) continue;
            const auto k0 = cellOf(&wc[i * 3]);
            int64_t best = -1;
            for (int a = -1; a <= 1; a++)
                for (int b = -1; b <= 1; b++)
                    for (int c = -1; c <= 1; c++) {
                        auto it = grid.find({k0[0] + a, k0[1] + b, k0[2] + c});
                        if (it == grid.end()) continue;
                        for (int64_t j : it->second)
                            if ((size_t)j != i && !done[j] && near(i, (size_t)j) && (best < 0 || j < best)) best = j;
                    }
            if (best < 0) continue;
            done[i] = done[best] = 1;
            const int64_t ef = unmatched[i], other = unmatched[best];
            const int e = (int)(ef / 6), f = (int)(ef % 6), e1 = (int)(other / 6), f1 = (int)(other % 6);
            m.neig[(size_t)e * 6 + f] = e1;
            m.neigFc[(size_t)e * 6 + f] = f1;
            m.neig[(size_t)e1 * 6 + f1] = e;
            m.neigFc[(size_t)e1 * 6 + f1] = f;
            for (int d = 0; d < 3; d++) {
                // position of the shared face as seen from the other element
                const double sh = m.elFcCenter[(size_t)other * 3 + d] - m.elFcCenter[(size_t)ef * 3 + d];
                const double q = (L[d] > 0) ? L[d] * std::llround(sh / L[d]) : 0.0;
                m.neigShift[(size_t)e * 18 + f * 3 + d] = q;    // face of e seen from e1 = centre(e) + q
                m.neigShift[(size_t)e1 * 18 + f1 * 3 + d] = -q;
            }
            m.nPeriodic++;
        }
        std::vector<int64_t> still;
        for (size_t i = 0; i < nU; i++)
            if (!done[i]) still.push_back(unmatched[i]);
        unmatched.swap(still);
    }
    if (!unmatched.empty()) {
        const int64_t ef = *std::min_element(unmatched.begin(), unmatched.end());
        err = "open boundary face without a boundary condition: element " + std::to_string(ef / 6 + 1) +
              " face " + std::to_string(ef % 6 + 1) + " (" + std::to_string(unmatched.size()) + " such faces)";
        return FG_ERR_MESH;
    }
    return FG_OK;
}

// The reference face order, face and cell geometry and the device ordering (host path).
int finish_order_geometry(Mesh &m, const fg_mesh_opts &o, std::string &err) {
    const int nE = m.nElem;
    // reference face order: owner = first visited element (DP/buildLocalMesh.cu:263-313)
    m.fc2el.clear(); m.fc2elFc.clear(); m.boundCond.clear();
    m.fc2el.reserve((size_t)nE * 4); m.fc2elFc.reserve((size_t)nE * 4);
    std::vector<int32_t> fcShiftSrc;  // element-face slot that owns the face (for shifts)
    int maxF = 0;
    for (int e = 0; e < nE; e++) {
        const ElemType *et = elem_type_for_nodes(m.elNN[e]);
        maxF = std::max(maxF, et->nFaces);
        for (int f = 0; f < et->nFaces; f++) {
            const int e1 = m.neig[(size_t)e * 6 + f];
            if (e1 == -1 || e1 > e) {
                m.fc2el.push_back(e);
                m.fc2el.push_back(e1);
                m.fc2elFc.push_back(f);
                m.fc2elFc.push_back(e1 == -1 ? 0 : m.neigFc[(size_t)e * 6 + f]);
                m.boundCond.push_back(m.elBc[(size_t)e * 6 + f]);
                fcShiftSrc.push_back(e * 6 + f);
            }
        }
    }
    m.maxFaces = maxF;
    m.nFcs = (int)m.boundCond.size();
    const int nF = m.nFcs;
    m.nBoundary = 0;
    for (int f = 0; f < nF; f++) m.nBoundary += (m.boundCond[f] != 0);
    m.fcCenter.resize((size_t)nF * 3);
    m.n.resize((size_t)nF * 3);
    m.nt1.resize((size_t)nF * 3);
    m.nt2.resize((size_t)nF * 3);
    m.area.resize(nF);
    m.nbShift.assign((size_t)nF * 3, 0.0);
    for (int f = 0; f < nF; f++) {
        const int e = m.fc2el[2 * f], lf = m.fc2elFc[2 * f];
        const ElemType *et = elem_type_for_nodes(m.elNN[e]);
        double x[4], y[4], z[4];
        const int cnt = et->faceNodeCount[lf];
        for (int i = 0; i < cnt; i++) {
            const int nd = m.elNodes[(size_t)e * 8 + et->geomNodes[lf][i]];
            x[i] = m.nodes[(size_t)nd * 3 + 0];
            y[i] = m.nodes[(size_t)nd * 3 + 1];
            z[i] = m.nodes[(size_t)nd * 3 + 2];
        }
        normal_vector(x, y, z, &m.n[(size_t)f * 3]);
        tangent_vectors(x, y, z, &m.n[(size_t)f * 3], &m.nt1[(size_t)f * 3], &m.nt2[(size_t)f * 3]);
        m.area[f] = fan_area(cnt, x, y, z);
        for (int d = 0; d < 3; d++) {
            m.fcCenter[(size_t)f * 3 + d] = m.elFcCenter[(size_t)e * 18 + lf * 3 + d];
            m.nbShift[(size_t)f * 3 + d] = m.neigShift[(size_t)fcShiftSrc[f] * 3 + d];
        }
    }
    // volumes by tetra split from node 0 (DP/meshProperties.cu:102-137)
    m.volume.resize(nE);
    for (int e = 0; e < nE; e++) {
        const ElemType *et = elem_type_for_nodes(m.elNN[e]);
        const double *p0 = &m.nodes[(size_t)m.elNodes[(size_t)e * 8 + 0] * 3];
        double vol = 0.0;
        for (int t = 0; t < et->volTets; t++) {
            double dx[3], dy[3], dz[3];
            for (int i = 0; i < 3; i++) {
                const double *pi = &m.nodes[(size_t)m.elNodes[(size_t)e * 8 + et->volNodes[t][i]] * 3];
                dx[i] = pi[0] - p0[0];
                dy[i] = pi[1] - p0[1];
                dz[i] = pi[2] - p0[2];
            }
            const double c0 = dy[0] * dz[1] - dz[0] * dy[1];
            const double c1 = dz[0] * dx[1] - dx[0] * dz[1];
            const double c2 = dx[0] * dy[1] - dy[0] * dx[1];
            vol += (c0 * dx[2] + c1 * dy[2] + c2 * dz[2]) / 6.0;
        }
        m.volume[e] = vol;
        if (!(vol > 0.0)) {
            err = "element " + std::to_string(e + 1) + " has non-positive volume (inverted node order)";
            return FG_ERR_MESH;
        }
    }
    // device ordering
    m.new2old.resize(nE);
    std::iota(m.new2old.begin(), m.new2old.end(), 0);
    if (o.renumber == FG_RENUMBER_MORTON) {
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int e = 0; e < nE; e++)
            for (int d = 0; d < 3; d++) {
                lo[d] = std::min(lo[d], m.cellCenter[(size_t)e * 3 + d]);
                hi[d] = std::max(hi[d], m.cellCenter[(size_t)e * 3 + d]);
            }
        std::vector<uint64_t> key(nE);
        for (int e = 0; e < nE; e++) {
            uint32_t q[3];
            for (int d = 0; d < 3; d++) {
                const double span = hi[d] - lo[d];
                const double t = span > 0 ? (m.cellCenter[(size_t)e * 3 + d] - lo[d]) / span : 0.0;
                q[d] = (uint32_t)std::min(2097151.0, std::max(0.0, t * 2097151.0));
            }
            key[e] = morton3(q[0], q[1], q[2]);
        }
        std::stable_sort(m.new2old.begin(), m.new2old.end(), [&](int a, int b) { return key[a] < key[b]; });
    } else if (o.renumber == FG_RENUMBER_RCM) {
        // reverse Cuthill-McKee on the cell adjacency graph, per connected component
        std::vector<int> deg(nE, 0);
        for (int e = 0; e < nE; e++)
            for (int f = 0; f < 6; f++) deg[e] += (m.neig[(size_t)e * 6 + f] >= 0);
        std::vector<char> vis(nE, 0);
        std::vector<int> order;
        order.reserve(nE);
        std::vector<int> byDeg(nE);
        std::iota(byDeg.begin(), byDeg.end(), 0);
        std::stable_sort(byDeg.begin(), byDeg.end(), [&](int a, int b) { return deg[a] < deg[b]; });
        for (int s0 : byDeg) {
            if (vis[s0]) continue;
            std::queue<int> q;
            q.push(s0);
            vis[s0] = 1;
            while (!q.empty()) {
                const int e = q.front();
                q.pop();
                order.push_back(e);
                int nb[6], k = 0;
                for (int f = 0; f < 6; f++) {
                    const int e1 = m.neig[(size_t)e * 6 + f];
                    if (e1 >= 0 && !vis[e1]) { vis[e1] = 1; nb[k++] = e1; }
                }
                std::sort(nb, nb + k, [&](int a, int b) { return deg[a] < deg[b]; });
                for (int i = 0; i < k; i++) q.push(nb[i]);
            }
        }
        std::reverse(order.begin(), order.end());
        m.new2old = order;
    }
    m.old2new.resize(nE);
    for (int i = 0; i < nE; i++) m.old2new[m.new2old[i]] = i;
    return FG_OK;
}

}  // namespace fg
