// partition.cpp -- see partition.h.
#include "partition.h"

#include <algorithm>
#include <array>
#include <map>
#include <stdexcept>

namespace dgh {

std::vector<int> slab_partition(const int n[3], int nparts, int axis)
{
    if (nparts < 1 || axis < 0 || axis > 2 || n[0] < 1 || n[1] < 1 || n[2] < 1)
        throw std::invalid_argument("bad slab partition");
    const int ne = n[0] * n[1] * n[2];
    std::vector<int> part(ne);
    for (int e = 0; e < ne; ++e) {
        const int c[3] = {e % n[0], (e / n[0]) % n[1], e / (n[0] * n[1])};
        part[e] = static_cast<int>(static_cast<long long>(c[axis]) * nparts / n[axis]);
    }
    return part;
}

LocalMesh partition_mesh(const BoxMesh& g, const std::vector<int>& elem_part, int part)
{
    const int ne = g.nelem;
    if (static_cast<int>(elem_part.size()) != ne) throw std::invalid_argument("partition size mismatch");
    // boundary flag of every element, from the faces
    std::vector<char> boundary(ne, 0);
    for (int i = 0; i < g.nface; ++i) {
        const unsigned* r = &g.faces[static_cast<size_t>(i) * 8];
        const int eL = static_cast<int>(r[1]), eR = static_cast<int>(r[5]);
        if (elem_part[eL] != elem_part[eR]) boundary[eL] = boundary[eR] = 1;
    }
    // local ids of every element on its own part: interior first, then boundary
    std::map<int, int> count_interior;
    for (int e = 0; e < ne; ++e)
        if (!boundary[e]) ++count_interior[elem_part[e]];
    std::map<int, int> next_interior, next_boundary;
    std::vector<int> local_on_owner(ne);
    for (int e = 0; e < ne; ++e) {
        const int p = elem_part[e];
        local_on_owner[e] = boundary[e] ? count_interior[p] + next_boundary[p]++ : next_interior[p]++;
    }
    LocalMesh out;
    std::vector<int> owned;
    for (int e = 0; e < ne; ++e)
        if (elem_part[e] == part) owned.push_back(e);
    std::stable_sort(owned.begin(), owned.end(), [&](int a, int b) { return boundary[a] < boundary[b]; });
    out.nowned = static_cast<int>(owned.size());
    out.ninterior = count_interior[part];
    std::vector<int> ghosts;
    for (int i = 0; i < g.nface; ++i) {
        const unsigned* r = &g.faces[static_cast<size_t>(i) * 8];
        const int eL = static_cast<int>(r[1]), eR = static_cast<int>(r[5]);
        if (elem_part[eL] == part && elem_part[eR] != part) ghosts.push_back(eR);
        if (elem_part[eR] == part && elem_part[eL] != part) ghosts.push_back(eL);
    }
    std::sort(ghosts.begin(), ghosts.end());
    ghosts.erase(std::unique(ghosts.begin(), ghosts.end()), ghosts.end());
    out.global_elem = owned;
    out.global_elem.insert(out.global_elem.end(), ghosts.begin(), ghosts.end());
    for (int e : ghosts) {
        out.ghost_rank.push_back(elem_part[e]);
        out.ghost_elem.push_back(local_on_owner[e]);
    }
    std::vector<int> local_of(ne, -1);
    for (size_t l = 0; l < out.global_elem.size(); ++l) local_of[out.global_elem[l]] = static_cast<int>(l);
    // nodes of the local elements, in global node order
    std::vector<int> node_local(static_cast<size_t>(g.nnode), -1);
    std::vector<int> nodes;
    for (int e : out.global_elem)
        for (int l = 0; l < 8; ++l) nodes.push_back(static_cast<int>(g.e2n[static_cast<size_t>(e) * 8 + l]));
    std::sort(nodes.begin(), nodes.end());
    nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
    BoxMesh& m = out.mesh;
    m.nnode = static_cast<int>(nodes.size());
    m.coords.resize(nodes.size() * 3);
    for (size_t i = 0; i < nodes.size(); ++i) {
        node_local[nodes[i]] = static_cast<int>(i);
        for (int a = 0; a < 3; ++a) m.coords[i * 3 + a] = g.coords[static_cast<size_t>(nodes[i]) * 3 + a];
    }
    m.nelem = static_cast<int>(out.global_elem.size());
    m.e2n.resize(static_cast<size_t>(m.nelem) * 8);
    for (int l = 0; l < m.nelem; ++l)
        for (int k = 0; k < 8; ++k)
            m.e2n[static_cast<size_t>(l) * 8 + k] =
                static_cast<unsigned>(node_local[g.e2n[static_cast<size_t>(out.global_elem[l]) * 8 + k]]);
    for (int i = 0; i < g.nface; ++i) {
        const unsigned* r = &g.faces[static_cast<size_t>(i) * 8];
        const int eL = static_cast<int>(r[1]), eR = static_cast<int>(r[5]);
        if (elem_part[eL] != part && elem_part[eR] != part) continue;
        const unsigned row[8] = {static_cast<unsigned>(elem_part[eL]), static_cast<unsigned>(local_of[eL]), r[2], r[3],
                                 static_cast<unsigned>(elem_part[eR]), static_cast<unsigned>(local_of[eR]), r[6], r[7]};
        m.faces.insert(m.faces.end(), row, row + 8);
    }
    m.nface = static_cast<int>(m.faces.size() / 8);
    return out;
}

std::string make_halo_plan(const MeshView& mv, const int* ghost_elem, HaloPlan& out)
{
    out = HaloPlan{};
    const int nowned = mv.nowned < 0 ? mv.nelem : mv.nowned;
    struct Slice {
        std::array<int, 3> key;  // left side: rank, local id on that rank, face
        int peer, se, sf, re, rf;
    };
    std::vector<Slice> s;
    for (int i = 0; i < mv.nface; ++i) {
        const unsigned* r = &mv.faces[static_cast<size_t>(i) * 8];
        // unsigned comparisons: a negative entry is a huge one, not a small one
        if (r[1] >= static_cast<unsigned>(mv.nelem) || r[5] >= static_cast<unsigned>(mv.nelem) || r[2] > 5u ||
            r[6] > 5u)
            return "face " + std::to_string(i) + " has an out-of-range entry";
        const int eL = static_cast<int>(r[1]), fL = static_cast<int>(r[2]);
        const int eR = static_cast<int>(r[5]), fR = static_cast<int>(r[6]);
        const bool gL = eL >= nowned, gR = eR >= nowned;
        if (gL == gR) continue;  // owned-owned (local) or ghost-ghost (not ours)
        const int ghost = gL ? eL : eR, own = gL ? eR : eL;
        const int peer = mv.elem_rank ? mv.elem_rank[ghost] : mv.rank;
        if (peer == mv.rank) return "ghost element " + std::to_string(ghost) + " is owned by this rank";
        const int gid = ghost_elem ? ghost_elem[ghost - nowned] : -1;
        if (gid < 0) return "ghost element " + std::to_string(ghost) + " has no owner-local id";
        Slice x;
        x.key = gL ? std::array<int, 3>{peer, gid, fL} : std::array<int, 3>{mv.rank, own, fL};
        x.peer = peer;
        x.se = own;
        x.sf = gL ? fR : fL;
        x.re = ghost;
        x.rf = gL ? fL : fR;
        s.push_back(x);
    }
    std::sort(s.begin(), s.end(), [](const Slice& a, const Slice& b) {
        return a.peer != b.peer ? a.peer < b.peer : a.key < b.key;
    });
    for (size_t i = 0; i < s.size(); ++i) {
        if (out.peer_rank.empty() || out.peer_rank.back() != s[i].peer) {
            out.peer_rank.push_back(s[i].peer);
            out.peer_offset.push_back(static_cast<int>(i));
            out.peer_count.push_back(0);
        }
        ++out.peer_count.back();
        out.send_elem.push_back(s[i].se);
        out.send_face.push_back(s[i].sf);
        out.recv_elem.push_back(s[i].re);
        out.recv_face.push_back(s[i].rf);
    }
    return "";
}

}  // namespace dgh
