// mesh.h -- host-side mesh handling: periodic-box generation in the
// reference's mesh format, and the preparation of the device tables (geometry
// classes, periodic face-gather table) from interior_faces.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace dgh {

// The reference's in-memory mesh (src/mesh/mesh.h:280-310): node_coords
// [nnode][3], elem_to_node_IDs [ne][8], interior_faces [nface][8] =
// (rankL, elemL, faceL, orientL, rankR, elemR, faceR, orientR).
struct MeshView {
    int nnode = 0, nelem = 0, nface = 0, rank = 0;
    const double* coords = nullptr;
    const unsigned* e2n = nullptr;
    const unsigned* faces = nullptr;
    const int* tag = nullptr;  // optional [ne]: elements with different tags get different geometry classes
    // partitioned meshes: elements [nowned, nelem) are ghosts (copies of other
    // ranks' elements whose boundary slices arrive by halo exchange), and
    // elem_rank[e] is the owner of local element e; nowned < 0: no ghosts
    int nowned = -1;
    const int* elem_rank = nullptr;
};

struct BoxMesh {
    std::vector<double> coords;
    std::vector<unsigned> e2n;
    std::vector<unsigned> faces;
    int nnode = 0, nelem = 0, nface = 0;
};

// Uniform periodic box, element id i + n0*(j + n1*k); see dg_mesh_periodic_box.
BoxMesh make_periodic_box(const int n[3], const double x0[3], const double len[3], unsigned rotate_seed);

// One affine geometry shared by a set of elements.
struct GeoClass {
    double J[9];      // dx_i / dxi_j
    double JD[9];     // ijac(d, j) * djac  (contravariant flux transform)
    double djac;      // det J
    double inv_djac;  // 1 / det J
    double N[6][3];   // unnormalised outward normal of each reference face
    // the numerical fluxes' per-face normal data (base/functions.cpp:40-49,
    // euler/functions.cpp:309-311): |N|, N / |N| and N * (1 / |N|)
    double nmag[6];
    double nhat[6][3];
    double nunit[6][3];
};

// Everything the kernels need besides the state.
struct PreparedMesh {
    int ne = 0, m = 0;
    int nowned = 0;                    // elements [nowned, ne) are ghosts
    std::vector<int> geo_class;        // [ne]
    std::vector<GeoClass> classes;
    std::vector<int> conn;             // [ne][6][2]: neighbour element, packed (fn | isL<<3 | code<<4)
    std::vector<uint8_t> cmap;         // [ncodes][m*m]: own canonical face point -> neighbour's
    int ncodes = 0;
    std::vector<double> X0;            // [ne][3] coordinates of local node 0
    double volume = 0.0;               // sum of element volumes
    double hmin = 0.0;                 // smallest element edge length
    // General (trilinear, non-parallelepiped) geometry: set when some element
    // is not affine.  Every element then carries per-point tables, as the
    // reference's per-quadrature-point helpers do (helpers.cpp:5-51,
    // 380-500), and the affine classes are unused (one placeholder class).
    bool general = false;
    std::vector<double> gnodes;        // [ne][8][3] node coordinates
    std::vector<double> gjd;           // [ne][9][m^3] ijac(d, j) * djac at the volume GL points
    std::vector<double> gN;            // [nowned][6][3][m*m] the left element's face normal N at each own face point
    std::vector<double> elem_h;        // [ne] shortest edge of each element
};

// Validates the mesh and builds the tables for face grids of m x m points.
// Returns an empty string on success, else the reason (the caller maps it to
// DG_ERR_ARG / DG_ERR_UNSUPPORTED by the prefix "unsupported:").
std::string prepare_mesh(const MeshView& mv, int m, PreparedMesh& out);

}  // namespace dgh
