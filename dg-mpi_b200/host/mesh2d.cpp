// mesh2d.cpp -- periodic quadrilateral boxes in the reference's mesh form
// (the 2D counterpart of the hexahedral box generator of mesh.cpp).
//
// Nodes are not shared across the periodic boundary; periodicity lives in
// interior_faces.  Local faces follow get_local_nodes_on_face_quadrilateral
// (src/numerics/basis/shape.cpp:125-152): face 0 = nodes 0-1, 1 = 1-3,
// 2 = 3-2, 3 = 2-0, each traversed counter-clockwise around the element, so
// two neighbours traverse their shared edge in opposite directions: the left
// side takes orientation 0 and the right side orientation 1
// (get_face_pts_order_wrt_orient0_quadrilateral, shape.cpp:43-66).
#include <cstring>
#include <exception>
#include <vector>

#include "../../include/dg_b200.h"

namespace {

// reference positions of the four nodes (x fastest)
constexpr int kRefX[4] = {-1, 1, -1, 1}, kRefY[4] = {-1, -1, 1, 1};

// node k of an element whose local frame is rotated by r quarter turns
// counter-clockwise: the corner (0 BL, 1 BR, 2 TL, 3 TR) at the rotated
// reference position of node k
int rotated_corner(int k, int r)
{
    int x = kRefX[k], y = kRefY[k];
    for (int i = 0; i < r; ++i) {
        const int t = x;
        x = -y;
        y = t;
    }
    return (x > 0 ? 1 : 0) + (y > 0 ? 2 : 0);
}

unsigned next_rand(unsigned& s)
{
    s = s * 1664525u + 1013904223u;
    return s >> 16;
}

}  // namespace

extern "C" int dg_mesh2d_periodic_box(const int n[2], const double x0[2], const double len[2], unsigned rotate_seed,
                                      int* nnode, double* node_coords, int* nelem, unsigned* elem_to_node_ids,
                                      int* nface, unsigned* interior_faces)
{
    if (!n || !x0 || !len || !nnode || !nelem || !nface) return DG_ERR_ARG;
    if (n[0] < 1 || n[1] < 1 || !(len[0] > 0.0) || !(len[1] > 0.0)) return DG_ERR_ARG;
    const long long ne = 1LL * n[0] * n[1];
    if (ne > (1LL << 28)) return DG_ERR_ARG;
    const int n0 = n[0], n1 = n[1];
    *nnode = (n0 + 1) * (n1 + 1);
    *nelem = static_cast<int>(ne);
    *nface = static_cast<int>(2 * ne);
    if (!node_coords && !elem_to_node_ids && !interior_faces) return DG_OK;
    if (!node_coords || !elem_to_node_ids || !interior_faces) return DG_ERR_ARG;
    try {
        for (int j = 0; j <= n1; ++j)
            for (int i = 0; i <= n0; ++i) {
                double* c = node_coords + 2 * (static_cast<size_t>(j) * (n0 + 1) + i);
                c[0] = x0[0] + len[0] * i / n0;
                c[1] = x0[1] + len[1] * j / n1;
            }
        std::vector<int> rot(static_cast<size_t>(ne), 0);
        unsigned s = rotate_seed;
        for (long long e = 0; e < ne; ++e) rot[e] = rotate_seed ? static_cast<int>(next_rand(s) & 3u) : 0;
        auto node = [&](int i, int j) { return static_cast<unsigned>(j * (n0 + 1) + i); };
        auto elem = [&](int i, int j) { return static_cast<unsigned>(((j + n1) % n1) * n0 + (i + n0) % n0); };
        for (int j = 0; j < n1; ++j)
            for (int i = 0; i < n0; ++i) {
                const unsigned e = elem(i, j);
                const unsigned corner[4] = {node(i, j), node(i + 1, j), node(i, j + 1), node(i + 1, j + 1)};
                for (int k = 0; k < 4; ++k) elem_to_node_ids[4 * e + k] = corner[rotated_corner(k, rot[e])];
            }
        // the local face of physical edge P (0 bottom, 1 right, 2 top, 3 left)
        auto local_face = [&](unsigned e, int P) { return static_cast<unsigned>((P - rot[e] + 4) % 4); };
        for (int j = 0; j < n1; ++j)
            for (int i = 0; i < n0; ++i) {
                const unsigned e = elem(i, j), ex = elem(i + 1, j), ey = elem(i, j + 1);
                unsigned* fx = interior_faces + 16 * static_cast<size_t>(e);
                const unsigned rx[8] = {0, e, local_face(e, 1), 0, 0, ex, local_face(ex, 3), 1};
                const unsigned ry[8] = {0, e, local_face(e, 2), 0, 0, ey, local_face(ey, 0), 1};
                std::memcpy(fx, rx, sizeof(rx));
                std::memcpy(fx + 8, ry, sizeof(ry));
            }
    } catch (const std::exception&) {
        return DG_ERR_NOMEM;
    }
    return DG_OK;
}
