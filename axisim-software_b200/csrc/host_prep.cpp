// host_prep.cpp -- multiblock packer, trellis / triangle mesh builders with
// boundary classification, agglomeration hierarchy, colouring and boundary
// defaults (host side, once per solve). Behaviour follows the reference
// files cited per routine; the code is this project's own.
#include "host_prep.hpp"

#include <algorithm>
#include <climits>
#include <cmath>
#include <memory>
#include <numeric>
#include <thread>
#include <stdexcept>
#include <unordered_map>

namespace axisim {

namespace {

constexpr double kPi = 3.14159265358979323846;

struct Node {
    double z, r;
};

struct Block {
    int nr = 0, nz = 0, offset = 0;
    std::vector<Node> nodes;  // (nr+1)*(nz+1), row I (radial), column J (axial)
    int edgeGroup[4] = {-1, -1, -1, -1};
    const Node& at(int I, int J) const { return nodes[(size_t)I * (nz + 1) + J]; }
    int cell(int i, int j) const { return offset + i * nz + j; }
};

// Cell-boundary coordinates of one zone (multiblock.h:59-80).
std::vector<double> zoneFaces(double length, int n, int grading, double coef, double start) {
    std::vector<double> d((size_t)n, length / n);
    if (grading == 1 && n > 1 && coef > 0.0 && coef != 1.0) {
        const double d0 = length * (coef - 1.0) / (std::pow(coef, n) - 1.0);
        for (int k = 0; k < n; k++) d[(size_t)k] = d0 * std::pow(coef, k);
    }
    std::vector<double> f;
    f.reserve((size_t)n + 1);
    double x = start;
    f.push_back(x);
    for (int k = 0; k < n; k++) {
        x += d[(size_t)k];
        f.push_back(x);
    }
    return f;
}

// Edge numbering West, East, South, North (multiblock.h:85).
void edgeEnds(const Block& b, int e, Node& s, Node& t) {
    switch (e) {
        case 0: s = b.at(0, 0); t = b.at(b.nr, 0); break;
        case 1: s = b.at(0, b.nz); t = b.at(b.nr, b.nz); break;
        case 2: s = b.at(0, 0); t = b.at(0, b.nz); break;
        default: s = b.at(b.nr, 0); t = b.at(b.nr, b.nz); break;
    }
}
int edgeLen(const Block& b, int e) { return e <= 1 ? b.nr : b.nz; }
int edgeLocalCell(const Block& b, int e, int k) {
    switch (e) {
        case 0: return k * b.nz;
        case 1: return k * b.nz + b.nz - 1;
        case 2: return k;
        default: return (b.nr - 1) * b.nz + k;
    }
}
void edgeSegment(const Block& b, int e, int k, Node& a, Node& c) {
    switch (e) {
        case 0: a = b.at(k, 0); c = b.at(k + 1, 0); break;
        case 1: a = b.at(k, b.nz); c = b.at(k + 1, b.nz); break;
        case 2: a = b.at(0, k); c = b.at(0, k + 1); break;
        default: a = b.at(b.nr, k); c = b.at(b.nr, k + 1); break;
    }
}

// Shoelace centroid and area of a quad (multiblock.h:272-295).
void quadGeometry(const Node (&p)[4], double& cz, double& cr, double& area) {
    double A = 0.0, Cz = 0.0, Cr = 0.0;
    for (int k = 0; k < 4; k++) {
        const Node& a = p[k];
        const Node& b = p[(k + 1) & 3];
        const double cross = a.z * b.r - b.z * a.r;
        A += cross;
        Cz += (a.z + b.z) * cross;
        Cr += (a.r + b.r) * cross;
    }
    A *= 0.5;
    if (std::fabs(A) < 1e-30) {
        cz = 0.25 * (p[0].z + p[1].z + p[2].z + p[3].z);
        cr = 0.25 * (p[0].r + p[1].r + p[2].r + p[3].r);
        area = 0.0;
        return;
    }
    cz = Cz / (6.0 * A);
    cr = Cr / (6.0 * A);
    area = std::fabs(A);
}

}  // namespace

PackedMesh buildMultiblock(const std::vector<BlockSpec>& spec, double tol, int defaultGroup, int& seamStatus) {
    seamStatus = 0;
    std::vector<Block> blocks(spec.size());
    int total = 0;
    for (size_t bi = 0; bi < spec.size(); bi++) {
        const BlockSpec& s = spec[bi];
        const std::vector<double> zf = zoneFaces(s.axialLength, s.axialCells, s.axialGrading, s.axialCoef, s.z0);
        const std::vector<double> rf = zoneFaces(s.radialLength, s.radialCells, s.radialGrading, s.radialCoef, s.r0);
        Block& b = blocks[bi];
        b.nz = s.axialCells;
        b.nr = s.radialCells;
        b.nodes.resize((size_t)(b.nr + 1) * (b.nz + 1));
        for (int I = 0; I <= b.nr; I++)
            for (int J = 0; J <= b.nz; J++) b.nodes[(size_t)I * (b.nz + 1) + J] = Node{zf[(size_t)J], rf[(size_t)I]};
        for (int e = 0; e < 4; e++) b.edgeGroup[e] = s.edgeGroup[e];
        b.offset = total;
        total += b.nr * b.nz;
    }

    // Conformal interfaces: fully coincident block edges (multiblock.h:220-251).
    struct Seam {
        int a, b, ea, eb;
        bool reversed;
    };
    std::vector<Seam> seams;
    const double tol2 = tol * tol;
    auto same = [&](const Node& p, const Node& q) {
        const double dz = p.z - q.z, dr = p.r - q.r;
        return dz * dz + dr * dr <= tol2;
    };
    bool bad = false;
    for (int a = 0; a < (int)blocks.size() && !bad; a++)
        for (int b = a + 1; b < (int)blocks.size() && !bad; b++)
            for (int ea = 0; ea < 4 && !bad; ea++)
                for (int eb = 0; eb < 4; eb++) {
                    Node as, ae, bs, be;
                    edgeEnds(blocks[(size_t)a], ea, as, ae);
                    edgeEnds(blocks[(size_t)b], eb, bs, be);
                    const bool aligned = same(as, bs) && same(ae, be);
                    const bool reversed = same(as, be) && same(ae, bs);
                    if (!aligned && !reversed) continue;
                    if (edgeLen(blocks[(size_t)a], ea) != edgeLen(blocks[(size_t)b], eb)) {
                        bad = true;
                        break;
                    }
                    seams.push_back(Seam{a, b, ea, eb, reversed});
                }
    if (bad) {
        seamStatus = 1;
        seams.clear();
    }

    PackedMesh m;
    m.nCells = total;
    m.cellCenterZ.assign((size_t)total, 0.0);
    m.cellCenterR.assign((size_t)total, 0.0);
    m.cellArea2D.assign((size_t)total, 0.0);
    m.cellVolume.assign((size_t)total, 0.0);
    for (const Block& b : blocks)
        for (int i = 0; i < b.nr; i++)
            for (int j = 0; j < b.nz; j++) {
                const Node q[4] = {b.at(i, j), b.at(i, j + 1), b.at(i + 1, j + 1), b.at(i + 1, j)};
                double cz, cr, area;
                quadGeometry(q, cz, cr, area);
                const size_t g = (size_t)b.cell(i, j);
                m.cellCenterZ[g] = cz;
                m.cellCenterR[g] = cr;
                m.cellArea2D[g] = area;
                m.cellVolume[g] = 2.0 * kPi * std::fabs(cr) * area;
            }

    std::vector<std::vector<int32_t>> cellFaces((size_t)total);
    auto emit = [&](int owner, int nb, const Node& a, const Node& c, int gid) {
        const int fid = (int)m.faceOwner.size();
        const double dz = c.z - a.z, dr = c.r - a.r;
        const double L = std::sqrt(dz * dz + dr * dr);
        const double fz = 0.5 * (a.z + c.z), fr = 0.5 * (a.r + c.r);
        double nz = (L > 0.0) ? dr / L : 0.0;
        double nr = (L > 0.0) ? -dz / L : 0.0;
        double tz, tr;
        if (nb >= 0) {
            tz = m.cellCenterZ[(size_t)nb] - m.cellCenterZ[(size_t)owner];
            tr = m.cellCenterR[(size_t)nb] - m.cellCenterR[(size_t)owner];
        } else {
            tz = fz - m.cellCenterZ[(size_t)owner];
            tr = fr - m.cellCenterR[(size_t)owner];
        }
        if (nz * tz + nr * tr < 0.0) {
            nz = -nz;
            nr = -nr;
        }
        m.faceOwner.push_back(owner);
        m.faceNeighbor.push_back(nb);
        m.faceNormalZ.push_back(nz);
        m.faceNormalR.push_back(nr);
        m.faceCenterZ.push_back(fz);
        m.faceCenterR.push_back(fr);
        m.faceArea.push_back(2.0 * kPi * std::fabs(fr) * L);
        m.faceBoundaryGroupID.push_back(gid);
        cellFaces[(size_t)owner].push_back(fid);
        if (nb >= 0) cellFaces[(size_t)nb].push_back(fid);
    };
    // Faces inside blocks: east then north of each cell (multiblock.h:382-394).
    for (const Block& b : blocks)
        for (int i = 0; i < b.nr; i++)
            for (int j = 0; j < b.nz; j++) {
                const int owner = b.cell(i, j);
                if (j + 1 < b.nz) emit(owner, b.cell(i, j + 1), b.at(i, j + 1), b.at(i + 1, j + 1), -1);
                if (i + 1 < b.nr) emit(owner, b.cell(i + 1, j), b.at(i + 1, j), b.at(i + 1, j + 1), -1);
            }
    // Interface faces (multiblock.h:397-414).
    std::vector<char> claimed(blocks.size() * 4, 0);
    for (const Seam& s : seams) {
        claimed[(size_t)s.a * 4 + s.ea] = 1;
        claimed[(size_t)s.b * 4 + s.eb] = 1;
        const Block& A = blocks[(size_t)s.a];
        const Block& B = blocks[(size_t)s.b];
        const int count = edgeLen(A, s.ea);
        for (int k = 0; k < count; k++) {
            Node n0, n1;
            edgeSegment(A, s.ea, k, n0, n1);
            const int kb = s.reversed ? (count - 1 - k) : k;
            emit(A.offset + edgeLocalCell(A, s.ea, k), B.offset + edgeLocalCell(B, s.eb, kb), n0, n1, -1);
        }
    }
    // External faces (multiblock.h:417-432).
    for (size_t bi = 0; bi < blocks.size(); bi++) {
        const Block& b = blocks[bi];
        for (int e = 0; e < 4; e++) {
            if (claimed[bi * 4 + (size_t)e]) continue;
            const int gid = b.edgeGroup[e] >= 0 ? b.edgeGroup[e] : defaultGroup;
            const int count = edgeLen(b, e);
            for (int k = 0; k < count; k++) {
                Node n0, n1;
                edgeSegment(b, e, k, n0, n1);
                emit(b.offset + edgeLocalCell(b, e, k), -1, n0, n1, gid);
            }
        }
    }
    m.nFaces = (int)m.faceOwner.size();
    m.cellFaceStart.assign((size_t)total + 1, 0);
    for (int c = 0; c < total; c++) m.cellFaceStart[(size_t)c + 1] = m.cellFaceStart[(size_t)c] + (int)cellFaces[(size_t)c].size();
    m.cellFaceIDs.reserve((size_t)m.cellFaceStart[(size_t)total]);
    for (int c = 0; c < total; c++)
        m.cellFaceIDs.insert(m.cellFaceIDs.end(), cellFaces[(size_t)c].begin(), cellFaces[(size_t)c].end());
    return m;
}

// ---------------- domain outline, trellis and triangle meshes ----------------

bool pointInsideDomain(const Outline& o, double z, double r) {
    bool inside = false;
    const int nv = (int)o.vz.size();
    for (size_t e = 0; e < o.e0.size(); e++) {
        const int v0 = o.e0[e], v1 = o.e1[e];
        if (v0 < 0 || v1 < 0 || v0 >= nv || v1 >= nv) continue;
        const double az = o.vz[(size_t)v0], ar = o.vr[(size_t)v0];
        const double bz = o.vz[(size_t)v1], br = o.vr[(size_t)v1];
        const bool straddles = (ar > r) != (br > r);
        if (!straddles) continue;
        const double zCross = az + (r - ar) * (bz - az) / (br - ar);
        if (z < zCross) inside = !inside;
    }
    return inside;
}

int groupAtPoint(const Outline& o, double z, double r, double tol) {
    int best = -1;
    double bestDist = tol;
    const int nv = (int)o.vz.size();
    for (size_t e = 0; e < o.e0.size(); e++) {
        if (o.group[e] < 0) continue;
        const int v0 = o.e0[e], v1 = o.e1[e];
        if (v0 < 0 || v1 < 0 || v0 >= nv || v1 >= nv) continue;
        // closestPointOnSegment + distance (math_func.cpp:75-80, 152-169)
        const double az = o.vz[(size_t)v0], ar = o.vr[(size_t)v0];
        const double abZ = o.vz[(size_t)v1] - az, abR = o.vr[(size_t)v1] - ar;
        const double apZ = z - az, apR = r - ar;
        const double ab2 = abZ * abZ + abR * abR;
        double qz = az, qr = ar;
        if (!(ab2 <= 1e-30)) {
            double t = (apZ * abZ + apR * abR) / ab2;
            t = std::clamp(t, 0.0, 1.0);
            qz = az + t * abZ;
            qr = ar + t * abR;
        }
        const double dz = qz - z, dr = qr - r;
        const double dist = std::sqrt(dz * dz + dr * dr);
        if (dist < bestDist) {
            bestDist = dist;
            best = o.group[e];
        }
    }
    return best;
}

void classifyBoundaryFaces(PackedMesh& m, const Outline& o, double L, double R) {
    const double matchTol = 1e-4 * std::max(std::max(L, R), 1.0);
    for (int f = 0; f < m.nFaces; f++) {
        if (m.faceNeighbor[(size_t)f] >= 0) continue;
        m.faceBoundaryGroupID[(size_t)f] = groupAtPoint(o, m.faceCenterZ[(size_t)f], m.faceCenterR[(size_t)f], matchTol);
    }
}

PackedMesh buildTrellis(const std::vector<double>& zL, const std::vector<double>& rL, const std::vector<int>& zCells,
                        const std::vector<int>& rCells, const Outline& o, double L, double R, int nz, int nr,
                        int& seamStatus) {
    std::vector<BlockSpec> blocks;
    if (zL.size() >= 2 && rL.size() >= 2) {
        for (size_t i = 0; i + 1 < zL.size(); i++)
            for (size_t j = 0; j + 1 < rL.size(); j++) {
                const double cz = 0.5 * (zL[i] + zL[i + 1]), cr = 0.5 * (rL[j] + rL[j + 1]);
                if (!pointInsideDomain(o, cz, cr)) continue;
                BlockSpec b;
                b.z0 = zL[i];
                b.r0 = rL[j];
                b.axialLength = zL[i + 1] - zL[i];
                b.axialCells = std::max(zCells[i], 1);
                b.radialLength = rL[j + 1] - rL[j];
                b.radialCells = std::max(rCells[j], 1);
                blocks.push_back(b);
            }
    }
    if (blocks.empty()) {
        BlockSpec b;
        b.axialLength = L;
        b.axialCells = std::max(nz, 1);
        b.radialLength = R;
        b.radialCells = std::max(nr, 1);
        blocks.push_back(b);
    }
    // trellis blocks share full edges: every seam is conformal
    PackedMesh m = buildMultiblock(blocks, std::max(L, R) * 1e-6, -1, seamStatus);
    classifyBoundaryFaces(m, o, L, R);
    return m;
}

PackedMesh buildTriangleMesh(const std::vector<double>& pz, const std::vector<double>& pr,
                             const std::vector<int32_t>& tri, const Outline& o, double L, double R) {
    constexpr double kPi = 3.14159265358979323846;
    const int T = (int)(tri.size() / 3);
    const int P = (int)pz.size();
    PackedMesh m;
    m.nCells = T;
    m.cellCenterZ.resize((size_t)T);
    m.cellCenterR.resize((size_t)T);
    m.cellArea2D.resize((size_t)T);
    m.cellVolume.resize((size_t)T);
    for (int c = 0; c < T; c++) {
        const int v[3] = {tri[3 * (size_t)c], tri[3 * (size_t)c + 1], tri[3 * (size_t)c + 2]};
        for (int k = 0; k < 3; k++)
            if (v[k] < 0 || v[k] >= P) throw std::runtime_error("triangle vertex out of range");
        const double az = pz[(size_t)v[0]], ar = pr[(size_t)v[0]];
        const double bz = pz[(size_t)v[1]], br = pr[(size_t)v[1]];
        const double dz_ = pz[(size_t)v[2]], dr_ = pr[(size_t)v[2]];
        m.cellCenterZ[(size_t)c] = (az + bz + dz_) / 3.0;   // triangleCentroid (mesh.cpp:1549-1554)
        m.cellCenterR[(size_t)c] = (ar + br + dr_) / 3.0;
        const double dz1 = bz - az, dr1 = br - ar, dz2 = dz_ - az, dr2 = dr_ - ar;
        m.cellArea2D[(size_t)c] = 0.5 * std::abs(dz1 * dr2 - dr1 * dz2);  // triangleArea2D
        m.cellVolume[(size_t)c] = 2.0 * kPi * m.cellCenterR[(size_t)c] * m.cellArea2D[(size_t)c];
    }
    std::unordered_map<int64_t, int32_t> edgeToFace;
    edgeToFace.reserve((size_t)T * 2);
    std::vector<int32_t> uses;
    m.cellFaceStart.assign((size_t)T + 1, 0);
    m.cellFaceIDs.reserve((size_t)T * 3);
    auto addEdge = [&](int c, int v0, int v1) {
        const int64_t key = (int64_t)std::min(v0, v1) * P + std::max(v0, v1);
        auto it = edgeToFace.find(key);
        if (it == edgeToFace.end()) {
            const double p0z = pz[(size_t)v0], p0r = pr[(size_t)v0], p1z = pz[(size_t)v1], p1r = pr[(size_t)v1];
            const double fz = 0.5 * (p0z + p1z), fr = 0.5 * (p0r + p1r);
            const double dz = p1z - p0z, dr = p1r - p0r;
            const double len = std::sqrt(dz * dz + dr * dr);
            double nzv = dr, nrv = -dz;
            const double mag = std::sqrt(nzv * nzv + nrv * nrv);
            if (mag > 1e-30) {
                nzv /= mag;
                nrv /= mag;
            }
            const double tz = fz - m.cellCenterZ[(size_t)c], tr = fr - m.cellCenterR[(size_t)c];
            if (nzv * tz + nrv * tr < 0.0) {
                nzv *= -1.0;
                nrv *= -1.0;
            }
            const int32_t id = m.nFaces++;
            m.faceOwner.push_back(c);
            m.faceNeighbor.push_back(-1);
            m.faceBoundaryGroupID.push_back(-1);
            m.faceCenterZ.push_back(fz);
            m.faceCenterR.push_back(fr);
            m.faceArea.push_back(2.0 * kPi * fr * len);
            m.faceNormalZ.push_back(nzv);
            m.faceNormalR.push_back(nrv);
            uses.push_back(1);
            edgeToFace.emplace(key, id);
            m.cellFaceIDs.push_back(id);
        } else {
            const int32_t id = it->second;
            if (++uses[(size_t)id] > 2) throw std::runtime_error("an edge is shared by more than two triangles");
            m.faceNeighbor[(size_t)id] = c;
            m.cellFaceIDs.push_back(id);
        }
    };
    for (int c = 0; c < T; c++) {
        const int v0 = tri[3 * (size_t)c], v1 = tri[3 * (size_t)c + 1], v2 = tri[3 * (size_t)c + 2];
        addEdge(c, v0, v1);
        addEdge(c, v1, v2);
        addEdge(c, v2, v0);
        m.cellFaceStart[(size_t)c + 1] = (int32_t)m.cellFaceIDs.size();
    }
    classifyBoundaryFaces(m, o, L, R);
    return m;
}

GridLevel finestLevel(int nCells, int nFaces, const int32_t* cfs, const int32_t* cfi, const int32_t* owner,
                      const int32_t* neighbor) {
    GridLevel g;
    g.nCells = nCells;
    g.faceStart.assign(cfs, cfs + nCells + 1);
    g.faceNeighbor.resize((size_t)cfs[nCells]);
    parallelFor(nCells, [&](int c0, int c1) {
        for (int c = c0; c < c1; c++)
            for (int k = cfs[c]; k < cfs[c + 1]; k++) {
                const int f = cfi[k];
                int nb = -1;
                if (f >= 0 && f < nFaces) {
                    if (owner[f] == c) nb = neighbor[f];
                    else if (neighbor[f] == c) nb = owner[f];
                }
                g.faceNeighbor[(size_t)k] = nb;
            }
    });
    return g;
}

namespace {

// Greedy breadth-first aggregates of up to four cells, singletons merged into
// their smallest neighbouring aggregate, ids compacted by first appearance
// (multigrid.cu:79-194).
int aggregate(const GridLevel& fine, std::vector<int32_t>& c2c) {
    constexpr int target = 4;
    const int N = fine.nCells;
    c2c.assign((size_t)N, -1);
    int nAgg = 0;
    int members[target];
    for (int n = 0; n < N; n++) {
        if (c2c[(size_t)n] >= 0) continue;
        const int c = nAgg++;
        c2c[(size_t)n] = c;
        int count = 0;
        members[count++] = n;
        for (int m = 0; m < count && count < target; m++) {
            const int cell = members[m];
            for (int k = fine.faceStart[(size_t)cell]; k < fine.faceStart[(size_t)cell + 1] && count < target; k++) {
                const int nb = fine.faceNeighbor[(size_t)k];
                if (nb < 0 || c2c[(size_t)nb] >= 0) continue;
                c2c[(size_t)nb] = c;
                members[count++] = nb;
            }
        }
    }
    std::vector<int> size((size_t)nAgg, 0);
    for (int n = 0; n < N; n++) size[(size_t)c2c[(size_t)n]]++;
    for (int n = 0; n < N; n++) {
        const int c = c2c[(size_t)n];
        if (size[(size_t)c] != 1) continue;
        int best = -1, bestSize = 0;
        for (int k = fine.faceStart[(size_t)n]; k < fine.faceStart[(size_t)n + 1]; k++) {
            const int nb = fine.faceNeighbor[(size_t)k];
            if (nb < 0) continue;
            const int cn = c2c[(size_t)nb];
            if (cn == c) continue;
            if (best < 0 || size[(size_t)cn] < bestSize) {
                best = cn;
                bestSize = size[(size_t)cn];
            }
        }
        if (best < 0) continue;
        c2c[(size_t)n] = best;
        size[(size_t)best]++;
        size[(size_t)c] = 0;
    }
    std::vector<int> remap((size_t)nAgg, -1);
    int next = 0;
    for (int n = 0; n < N; n++) {
        int& r = remap[(size_t)c2c[(size_t)n]];
        if (r < 0) r = next++;
        c2c[(size_t)n] = r;
    }
    return next;
}

// Coarse CSR + fine slot -> coarse slot map (multigrid.cu:196-287): every
// distinct (coarse cell, coarse neighbour) pair met across an aggregate
// boundary, in ascending order of cell then neighbour, and for each fine slot
// the coarse slot of its pair. Each aggregate's members (a counting sort of
// the fine cells) give its boundary slots, a few dozen, which are sorted by
// neighbour in place, so the cost is linear in the slots; the order of equal
// pairs does not change the result.
GridLevel coarsen(GridLevel& fine) {
    GridLevel coarse;
    const int nC = aggregate(fine, fine.cellToCoarse);
    coarse.nCells = nC;
    const int N = fine.nCells;
    const std::vector<int32_t>& c2c = fine.cellToCoarse;
    std::vector<int32_t> mStart((size_t)nC + 1, 0), mList((size_t)N);
    for (int n = 0; n < N; n++) mStart[(size_t)c2c[(size_t)n] + 1]++;
    for (int c = 0; c < nC; c++) mStart[(size_t)c + 1] += mStart[(size_t)c];
    {
        std::vector<int32_t> fill(mStart.begin(), mStart.end() - 1);
        for (int n = 0; n < N; n++) mList[(size_t)fill[(size_t)c2c[(size_t)n]]++] = n;
    }
    // every aggregate's boundary slots as (coarse neighbour, fine slot) pairs,
    // stored at the aggregate's offset among all member slots, sorted by
    // neighbour in place; aggregates are independent, so they run in parallel
    struct Ref {
        int32_t cn, slot;
    };
    std::vector<int64_t> refStart((size_t)nC + 1, 0);
    parallelFor(nC, [&](int c0, int c1) {
        for (int c = c0; c < c1; c++) {
            int64_t d = 0;
            for (int q = mStart[(size_t)c]; q < mStart[(size_t)c + 1]; q++) {
                const int n = mList[(size_t)q];
                d += fine.faceStart[(size_t)n + 1] - fine.faceStart[(size_t)n];
            }
            refStart[(size_t)c + 1] = d;
        }
    });
    for (int c = 0; c < nC; c++) refStart[(size_t)c + 1] += refStart[(size_t)c];
    // scratch left uninitialised (every entry read is written first): fresh
    // zero-filled pages of this size cost more than the pass itself
    std::unique_ptr<Ref[]> refs(new Ref[(size_t)std::max<int64_t>(refStart[(size_t)nC], 1)]);
    std::vector<int32_t> nRef((size_t)nC), nUnique((size_t)nC + 1, 0);
    fine.fineSlotToCoarseSlot.resize((size_t)fine.nFaceRefs());
    parallelFor(nC, [&](int c0, int c1) {
        for (int c = c0; c < c1; c++) {
            Ref* b = refs.get() + refStart[(size_t)c];
            Ref* e = b;
            for (int q = mStart[(size_t)c]; q < mStart[(size_t)c + 1]; q++) {
                const int n = mList[(size_t)q];
                for (int k = fine.faceStart[(size_t)n]; k < fine.faceStart[(size_t)n + 1]; k++) {
                    fine.fineSlotToCoarseSlot[(size_t)k] = -1;  // internal and boundary slots stay -1
                    const int nb = fine.faceNeighbor[(size_t)k];
                    if (nb < 0) continue;
                    const int cb = c2c[(size_t)nb];
                    if (cb != c) *e++ = Ref{cb, k};
                }
            }
            if (e - b > 32)
                std::sort(b, e, [](const Ref& x, const Ref& y) { return x.cn < y.cn; });
            else
                for (Ref* i = b + 1; i < e; i++)  // insertion sort by neighbour
                    for (Ref* j = i; j > b && (j - 1)->cn > j->cn; j--) std::swap(*(j - 1), *j);
            int u = 0;
            for (Ref* i = b; i < e; i++)
                if (i == b || i->cn != (i - 1)->cn) u++;
            nRef[(size_t)c] = (int32_t)(e - b);
            nUnique[(size_t)c + 1] = u;
        }
    });
    // the coarse CSR: distinct (coarse cell, coarse neighbour) pairs in
    // ascending order of cell then neighbour, and each fine slot's coarse slot
    for (int c = 0; c < nC; c++) nUnique[(size_t)c + 1] += nUnique[(size_t)c];
    coarse.faceStart.assign(nUnique.begin(), nUnique.end());
    coarse.faceNeighbor.resize((size_t)nUnique[(size_t)nC]);
    parallelFor(nC, [&](int c0, int c1) {
        for (int c = c0; c < c1; c++) {
            const Ref* b = refs.get() + refStart[(size_t)c];
            const Ref* e = b + nRef[(size_t)c];
            int pos = nUnique[(size_t)c] - 1;
            for (const Ref* i = b; i < e; i++) {
                if (i == b || i->cn != (i - 1)->cn) coarse.faceNeighbor[(size_t)++pos] = i->cn;
                fine.fineSlotToCoarseSlot[(size_t)i->slot] = pos;
            }
        }
    });
    return coarse;
}

}  // namespace

std::vector<GridLevel> buildHierarchy(GridLevel fine) {
    constexpr int minCoarseCells = 64;
    constexpr double maxShrinkRatio = 0.8;
    std::vector<GridLevel> levels;
    while (fine.nCells > minCoarseCells) {
        GridLevel coarse = coarsen(fine);
        if (coarse.nCells >= (int)(fine.nCells * maxShrinkRatio)) {
            fine.cellToCoarse.clear();
            fine.fineSlotToCoarseSlot.clear();
            break;
        }
        levels.push_back(std::move(fine));
        fine = std::move(coarse);
    }
    levels.push_back(std::move(fine));
    return levels;
}

std::vector<GridLevel> buildBatchHierarchy(const GridLevel& finest, const std::vector<int32_t>& caseStart,
                                           std::vector<std::vector<int32_t>>& terminal) {
    const int nCases = (int)caseStart.size() - 1;
    std::vector<std::vector<GridLevel>> per((size_t)nCases);
    size_t depth = 0;
    for (int c = 0; c < nCases; c++) {
        const int s = caseStart[(size_t)c], e = caseStart[(size_t)c + 1];
        GridLevel g;
        g.nCells = e - s;
        const int k0 = finest.faceStart[(size_t)s], k1 = finest.faceStart[(size_t)e];
        g.faceStart.resize((size_t)g.nCells + 1);
        for (int n = 0; n <= g.nCells; n++) g.faceStart[(size_t)n] = finest.faceStart[(size_t)(s + n)] - k0;
        g.faceNeighbor.resize((size_t)(k1 - k0));
        for (int k = k0; k < k1; k++) {
            const int nb = finest.faceNeighbor[(size_t)k];
            if (nb >= 0 && (nb < s || nb >= e)) throw std::runtime_error("a face connects two cases");
            g.faceNeighbor[(size_t)(k - k0)] = nb >= 0 ? nb - s : -1;
        }
        per[(size_t)c] = buildHierarchy(std::move(g));
        depth = std::max(depth, per[(size_t)c].size());
    }
    const int L = (int)depth;
    // cell and slot offsets of each case on each level (cases without the level add nothing)
    std::vector<std::vector<int64_t>> cellOff((size_t)L, std::vector<int64_t>((size_t)nCases + 1, 0));
    std::vector<std::vector<int64_t>> slotOff((size_t)L, std::vector<int64_t>((size_t)nCases + 1, 0));
    for (int l = 0; l < L; l++)
        for (int c = 0; c < nCases; c++) {
            const bool has = (int)per[(size_t)c].size() > l;
            const GridLevel* g = has ? &per[(size_t)c][(size_t)l] : nullptr;
            cellOff[(size_t)l][(size_t)c + 1] = cellOff[(size_t)l][(size_t)c] + (has ? g->nCells : 0);
            slotOff[(size_t)l][(size_t)c + 1] = slotOff[(size_t)l][(size_t)c] + (has ? g->nFaceRefs() : 0);
        }
    std::vector<GridLevel> out((size_t)L);
    terminal.assign((size_t)L, {});
    for (int l = 0; l < L; l++) {
        GridLevel& u = out[(size_t)l];
        if (cellOff[(size_t)l][(size_t)nCases] > INT32_MAX || slotOff[(size_t)l][(size_t)nCases] > INT32_MAX)
            throw std::runtime_error("batch too large");
        u.nCells = (int)cellOff[(size_t)l][(size_t)nCases];
        u.faceStart.assign((size_t)u.nCells + 1, 0);
        u.faceNeighbor.resize((size_t)slotOff[(size_t)l][(size_t)nCases]);
        const bool deepest = l == L - 1;
        if (!deepest) {
            u.cellToCoarse.assign((size_t)u.nCells, -1);
            u.fineSlotToCoarseSlot.assign(u.faceNeighbor.size(), -1);
        }
        for (int c = 0; c < nCases; c++) {
            if ((int)per[(size_t)c].size() <= l) continue;
            const GridLevel& g = per[(size_t)c][(size_t)l];
            const int co = (int)cellOff[(size_t)l][(size_t)c], so = (int)slotOff[(size_t)l][(size_t)c];
            for (int n = 0; n < g.nCells; n++) u.faceStart[(size_t)(co + n) + 1] = so + g.faceStart[(size_t)n + 1];
            for (int k = 0; k < g.nFaceRefs(); k++) {
                const int nb = g.faceNeighbor[(size_t)k];
                u.faceNeighbor[(size_t)(so + k)] = nb >= 0 ? nb + co : -1;
            }
            if (deepest) continue;
            if (g.isCoarsest()) {  // this case ends here: terminal cells, no coarse parent
                terminal[(size_t)l].push_back(co);
                terminal[(size_t)l].push_back(co + g.nCells);
                continue;
            }
            const int cco = (int)cellOff[(size_t)l + 1][(size_t)c], cso = (int)slotOff[(size_t)l + 1][(size_t)c];
            for (int n = 0; n < g.nCells; n++) u.cellToCoarse[(size_t)(co + n)] = g.cellToCoarse[(size_t)n] + cco;
            for (int k = 0; k < g.nFaceRefs(); k++) {
                const int t = g.fineSlotToCoarseSlot[(size_t)k];
                u.fineSlotToCoarseSlot[(size_t)(so + k)] = t >= 0 ? t + cso : -1;
            }
        }
    }
    return out;
}

int pickBlock(const std::vector<int>& candidates, const std::vector<double>& timeUs, int defaultIndex, double tol) {
    const int n = (int)std::min(candidates.size(), timeUs.size());
    auto ok = [&](int i) { return i >= 0 && i < n && std::isfinite(timeUs[(size_t)i]) && timeUs[(size_t)i] > 0.0; };
    int best = -1;
    for (int i = 0; i < n; i++)
        if (ok(i) && (best < 0 || timeUs[(size_t)i] < timeUs[(size_t)best])) best = i;
    if (best < 0) return (defaultIndex >= 0 && defaultIndex < n) ? defaultIndex : 0;  // nothing measured
    if (ok(defaultIndex) && timeUs[(size_t)defaultIndex] <= (1.0 + tol) * timeUs[(size_t)best]) return defaultIndex;
    return best;
}

namespace {

uint32_t spreadBits16(uint32_t v) {
    v &= 0xFFFFu;
    v = (v | (v << 8)) & 0x00FF00FFu;
    v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

// Open-addressing map from mesh cell to local index (key and value side by
// side, at most half full), cleared per tile by forgetting only the slots it
// used.
class LocalMap {
public:
    explicit LocalMap(int entries) {
        uint32_t size = 1024;
        while (size < 2u * (uint32_t)entries) size <<= 1;
        slots_.assign(size, Slot{-1, -1});
        mask_ = size - 1;
    }
    void clear() {
        for (uint32_t i : used_) slots_[i].key = -1;
        used_.clear();
    }
    bool insert(int32_t k) {  // true when k was not present
        const uint32_t i = slot(k);
        if (slots_[i].key == k) return false;
        slots_[i] = Slot{k, -1};
        used_.push_back(i);
        return true;
    }
    void set(int32_t k, int32_t v) { slots_[slot(k)].val = v; }
    int32_t get(int32_t k) const {
        const Slot& e = slots_[slot(k)];
        return e.key == k ? e.val : -1;
    }

private:
    struct Slot {
        int32_t key, val;
    };
    uint32_t slot(int32_t k) const {
        uint32_t i = ((uint32_t)k * 2654435761u) & mask_;
        while (slots_[i].key != -1 && slots_[i].key != k) i = (i + 1) & mask_;
        return i;
    }
    std::vector<Slot> slots_;
    std::vector<uint32_t> used_;
    uint32_t mask_ = 0;
};

struct TileRun {
    std::vector<int32_t> count, layerEnd, gid;
    std::vector<uint64_t> lnb;
};

// The tiles of curve positions [a, b), appended to out; false when one cell
// with its halo does not fit in cap local cells.
bool buildTileRun(const int32_t* order, int a, int b, int N, int W, const int32_t* nb, int S, int cap, LocalMap& map,
                  std::vector<int32_t>& cells, TileRun& out) {
    cells.assign(order + a, order + b);
    std::sort(cells.begin(), cells.end());
    map.clear();
    for (int32_t c : cells) map.insert(c);
    std::vector<int32_t> layerEnd((size_t)S + 1);
    layerEnd[0] = (int32_t)cells.size();
    bool fits = (int)cells.size() <= cap;
    size_t from = 0;
    for (int k = 1; k <= S && fits; k++) {
        const size_t to = cells.size();
        for (size_t i = from; i < to && fits; i++)
            for (int j = 0; j < W && fits; j++) {
                const int32_t m = nb[(size_t)j * N + cells[i]];
                if (m >= 0 && map.insert(m)) {
                    cells.push_back(m);
                    fits = (int)cells.size() <= cap;  // the map holds at most cap + 1 cells
                }
            }
        std::sort(cells.begin() + (std::ptrdiff_t)to, cells.end());
        from = to;
        layerEnd[(size_t)k] = (int32_t)cells.size();
    }
    if (!fits) {
        if (b - a <= 1) return false;
        const int mid = a + (b - a) / 2;
        return buildTileRun(order, a, mid, N, W, nb, S, cap, map, cells, out) &&
               buildTileRun(order, mid, b, N, W, nb, S, cap, map, cells, out);
    }
    for (size_t i = 0; i < cells.size(); i++) map.set(cells[i], (int32_t)i);
    const size_t inner = (size_t)layerEnd[(size_t)S - 1];
    for (size_t i = 0; i < cells.size(); i++) {
        uint64_t word = ~0ull;
        if (i < inner)
            for (int j = 0; j < W; j++) {
                const int32_t m = nb[(size_t)j * N + cells[i]];
                const uint64_t l = m >= 0 ? (uint64_t)(uint32_t)map.get(m) : 0xFFFFull;
                word = (word & ~(0xFFFFull << (16 * j))) | (l << (16 * j));
            }
        out.lnb.push_back(word);
    }
    out.count.push_back((int32_t)cells.size());
    out.layerEnd.insert(out.layerEnd.end(), layerEnd.begin(), layerEnd.end());
    out.gid.insert(out.gid.end(), cells.begin(), cells.end());
    return true;
}

}  // namespace

std::vector<int32_t> slotNeighbours(int N, int W, const int32_t* cfs, const int32_t* cfi, const int32_t* owner,
                                    const int32_t* neighbor) {
    std::vector<int32_t> nb((size_t)W * (size_t)std::max(N, 0));
    parallelFor(N, [&](int c0, int c1) {
        for (int c = c0; c < c1; c++) {
            const int k0 = cfs[c], deg = cfs[c + 1] - k0;
            for (int j = 0; j < W; j++) {
                int m = -1;
                if (j < deg) {
                    const int f = cfi[k0 + j];
                    if (owner[f] == c) m = neighbor[f];
                    else if (neighbor[f] == c) m = owner[f];
                }
                nb[(size_t)j * N + c] = m;
            }
        }
    });
    return nb;
}

SweepTiles buildSweepTiles(int N, int W, const int32_t* nb, const double* cz, const double* cr, int S, int cap,
                           int tileCells, const int32_t* caseStart, int nCases) {
    SweepTiles t;
    t.S = S;
    t.cap = cap;
    t.tileStart.assign(1, 0);
    if (N <= 0 || W < 1 || W > 4 || S < 1 || cap < 1 || cap >= 0xFFFF || tileCells < 1) return t;
    double z0 = cz[0], z1 = cz[0], r0 = cr[0], r1 = cr[0];
    for (int n = 1; n < N; n++) {
        z0 = std::min(z0, cz[n]);
        z1 = std::max(z1, cz[n]);
        r0 = std::min(r0, cr[n]);
        r1 = std::max(r1, cr[n]);
    }
    const double span = std::max(z1 - z0, r1 - r0);
    const double sc = span > 0.0 ? 65535.0 / span : 0.0;
    std::vector<uint32_t> key((size_t)N);
    parallelFor(N, [&](int b, int e) {
        for (int n = b; n < e; n++) {
            const double qz = (cz[n] - z0) * sc, qr = (cr[n] - r0) * sc;
            const uint32_t iz = qz >= 0.0 ? (uint32_t)std::min(qz, 65535.0) : 0u;
            const uint32_t ir = qr >= 0.0 ? (uint32_t)std::min(qr, 65535.0) : 0u;
            key[(size_t)n] = spreadBits16(iz) | (spreadBits16(ir) << 1);
        }
    });
    // cells by key: a counting sort on the top 16 bits (a 256 x 256 grid of
    // the bounding square; per-thread counts, so each bucket keeps ascending
    // cell order), then buckets of more than half a run by the whole key
    const int refine = std::max(64, tileCells / 2);
    std::vector<int32_t> order((size_t)N), tmp((size_t)N);
    {
        const unsigned hw = std::thread::hardware_concurrency();
        const int nt = std::max(1, std::min({(int)(hw ? hw : 1), 16, N / 16384}));
        const int chunk = (N + nt - 1) / nt;
        std::vector<int32_t> cnt((size_t)nt * 65536, 0);
        parallelFor(nt, [&](int t0, int t1) {
            for (int t = t0; t < t1; t++)
                for (int n = t * chunk, e = std::min(N, n + chunk); n < e; n++)
                    cnt[(size_t)t * 65536 + (key[(size_t)n] >> 16)]++;
        }, 1);
        // bucket starts, then each thread's first position in every bucket
        // (threads in order within a bucket), in row passes over the counts
        std::vector<int32_t> bucketStart(65537, 0), at(65536, 0);
        for (int t = 0; t < nt; t++)
            for (int d = 0; d < 65536; d++) at[(size_t)d] += cnt[(size_t)t * 65536 + d];
        for (int d = 0; d < 65536; d++) bucketStart[(size_t)d + 1] = bucketStart[(size_t)d] + at[(size_t)d];
        std::copy(bucketStart.begin(), bucketStart.end() - 1, at.begin());
        for (int t = 0; t < nt; t++)
            for (int d = 0; d < 65536; d++) {
                const int32_t c = cnt[(size_t)t * 65536 + d];
                cnt[(size_t)t * 65536 + d] = at[(size_t)d];
                at[(size_t)d] += c;
            }
        parallelFor(nt, [&](int t0, int t1) {
            for (int t = t0; t < t1; t++)
                for (int n = t * chunk, e = std::min(N, n + chunk); n < e; n++)
                    order[(size_t)cnt[(size_t)t * 65536 + (key[(size_t)n] >> 16)]++] = n;
        }, 1);
        parallelFor(65536, [&](int d0, int d1) {
            for (int d = d0; d < d1; d++) {
                int32_t* b = order.data() + bucketStart[(size_t)d];
                int32_t* e = order.data() + bucketStart[(size_t)d + 1];
                if (e - b > refine)
                    std::sort(b, e, [&](int32_t x, int32_t y) {
                        return key[(size_t)x] != key[(size_t)y] ? key[(size_t)x] < key[(size_t)y] : x < y;
                    });
            }
        }, 4096);
    }
    if (nCases > 1) {  // stable by case: the curve of case 0, then of case 1, ...
        std::vector<int32_t> at((size_t)nCases + 1);
        std::copy(caseStart, caseStart + nCases + 1, at.begin());
        for (int n = 0; n < N; n++) {
            const int32_t c = order[(size_t)n];
            const int k = (int)(std::upper_bound(caseStart, caseStart + nCases + 1, c) - caseStart) - 1;
            tmp[(size_t)at[(size_t)k]++] = c;
        }
        order.swap(tmp);
    }
    const int nRuns = (N + tileCells - 1) / tileCells;
    std::vector<TileRun> runs((size_t)nRuns);
    std::vector<char> ok((size_t)nRuns, 1);
    parallelFor(nRuns, [&](int rb, int re) {
        LocalMap map(cap + 1);
        std::vector<int32_t> cells;
        for (int r = rb; r < re; r++) {
            const int a = r * tileCells, b = std::min(N, a + tileCells);
            ok[(size_t)r] = buildTileRun(order.data(), a, b, N, W, nb, S, cap, map, cells, runs[(size_t)r]);
        }
    }, 4);
    for (char o : ok)
        if (!o) return t;
    // concatenate the runs in order, copies in parallel
    std::vector<size_t> tileOff((size_t)nRuns + 1, 0), localOff((size_t)nRuns + 1, 0);
    for (int r = 0; r < nRuns; r++) {
        tileOff[(size_t)r + 1] = tileOff[(size_t)r] + runs[(size_t)r].count.size();
        localOff[(size_t)r + 1] = localOff[(size_t)r] + runs[(size_t)r].gid.size();
    }
    const size_t nT = tileOff[(size_t)nRuns], nL = localOff[(size_t)nRuns];
    t.tileStart.resize(nT + 1);
    t.layerEnd.resize(nT * ((size_t)S + 1));
    t.gid.resize(nL);
    t.lnb.resize(nL);
    parallelFor(nRuns, [&](int r0, int r1) {
        for (int r = r0; r < r1; r++) {
            const TileRun& u = runs[(size_t)r];
            int32_t at = (int32_t)localOff[(size_t)r];
            for (size_t k = 0; k < u.count.size(); k++) {
                t.tileStart[tileOff[(size_t)r] + k] = at;
                at += u.count[k];
            }
            std::copy(u.layerEnd.begin(), u.layerEnd.end(), t.layerEnd.begin() + (std::ptrdiff_t)(tileOff[(size_t)r] * ((size_t)S + 1)));
            std::copy(u.gid.begin(), u.gid.end(), t.gid.begin() + (std::ptrdiff_t)localOff[(size_t)r]);
            std::copy(u.lnb.begin(), u.lnb.end(), t.lnb.begin() + (std::ptrdiff_t)localOff[(size_t)r]);
        }
    }, 4);
    t.tileStart[nT] = (int32_t)nL;
    return t;
}

int greedyColoring(const GridLevel& g, std::vector<int32_t>& color) {
    const int N = g.nCells;
    color.assign((size_t)N, -1);
    std::vector<int> stamp;
    int nColors = 0;
    for (int c = 0; c < N; c++) {
        for (int k = g.faceStart[(size_t)c]; k < g.faceStart[(size_t)c + 1]; k++) {
            const int nb = g.faceNeighbor[(size_t)k];
            if (nb < 0 || color[(size_t)nb] < 0) continue;
            const int cl = color[(size_t)nb];
            if (cl >= (int)stamp.size()) stamp.resize((size_t)cl + 1, -1);
            stamp[(size_t)cl] = c;
        }
        int pick = 0;
        while (pick < (int)stamp.size() && stamp[(size_t)pick] == c) pick++;
        color[(size_t)c] = pick;
        nColors = std::max(nColors, pick + 1);
    }
    return nColors;
}

uint8_t defaultBCType(int boundaryType, int variable) {
    // BCType: 0 DIRICHLET 1 NEUMANN 5 NONE; variables 0 u 1 v 2 p 3 T 4 C.
    // The scalars are Dirichlet at a velocity inlet, zero-gradient elsewhere.
    if (variable == 3 || variable == 4) return (boundaryType == 1) ? 0 : (boundaryType >= 0 && boundaryType <= 4) ? 1 : 5;
    switch (boundaryType) {
        case 1:  // VELOCITY_INLET
            return variable == 2 ? 1 : 0;
        case 2:  // PRESSURE_OUTLET
            return variable == 2 ? 0 : 1;
        case 0:  // WALL
            return variable == 2 ? 1 : 0;
        case 3:  // SYMMETRY: v Dirichlet 0, u and p zero-gradient
            return variable == 1 ? 0 : 1;
        case 4:  // FAR_FIELD
            return variable == 2 ? 1 : 0;
        default:
            return 5;
    }
}

bool variableEditable(int variable, int boundaryType) {
    const bool scalar = variable == 3 || variable == 4;
    switch (boundaryType) {
        case 0: return variable == 0 || variable == 1 || scalar;
        case 3: return false;
        case 4: return variable == 0 || variable == 1;
        case 1: return variable == 0 || variable == 1 || scalar;
        case 2: return variable == 2 || scalar;
        default: return false;
    }
}

}  // namespace axisim
