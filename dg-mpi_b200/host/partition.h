// partition.h -- host-side domain decomposition: element partitions of a mesh,
// rank-local meshes with ghost elements, and the halo-exchange plan that
// replaces MemoryNetwork::communicate_face_solution
// (src/memory/memory_network.cpp:55-175) and the ghost-face bookkeeping of
// the partitioned mesh reader (src/mesh/mesh.cpp:399-470).
#pragma once
#include <string>
#include <vector>

#include "mesh.h"

namespace dgh {

// element -> part for slabs along `axis` of an n0 x n1 x n2 box numbered
// i + n0*(j + n1*k): layer index * nparts / n[axis]
std::vector<int> slab_partition(const int n[3], int nparts, int axis);

// A rank-local mesh in the reference's in-memory format, with the ghost
// elements appended after the owned ones.  Owned elements are numbered
// interior first (no face shared with another part), then boundary elements,
// each in global order; ghost elements follow in global order.  Face rows
// reference local element ids and carry the owners' ranks in columns 0 and 4
// (as the reference's partitioned interior_faces do); only faces with at
// least one owned side are kept.
struct LocalMesh {
    BoxMesh mesh;                   // nodes, e2n, faces of owned + ghost elements
    int nowned = 0, ninterior = 0;
    std::vector<int> ghost_rank;    // [nghost] owning part of each ghost
    std::vector<int> ghost_elem;    // [nghost] its local id on that part
    std::vector<int> global_elem;   // [nowned + nghost] global element id
};

LocalMesh partition_mesh(const BoxMesh& global, const std::vector<int>& elem_part, int part);

// Who sends which boundary slices to whom.  Each face between an owned
// element and a ghost contributes one slice in each direction: this rank
// sends the coefficients of its element on that face and receives the
// ghost's.  Per peer, slices are ordered by the identity of the face's left
// side (its rank, its element's local id on that rank, its face), which both
// ranks of a face compute alike, so send slot i of one rank is receive slot i
// of the other.
struct HaloPlan {
    std::vector<int> peer_rank, peer_offset, peer_count;  // per peer, in slices
    std::vector<int> send_elem, send_face;                // [nslices] owned element / its face
    std::vector<int> recv_elem, recv_face;                // [nslices] ghost element (local id) / its face
};

// mv.nowned / mv.elem_rank describe the partition; ghost_elem[g] is the local
// id of ghost nowned+g on its owner.  Returns "" or the reason for rejecting.
std::string make_halo_plan(const MeshView& mv, const int* ghost_elem, HaloPlan& out);

}  // namespace dgh
