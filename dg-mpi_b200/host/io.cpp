// io.cpp -- the C ABI's mesh and solution files in the reference's HDF5
// schemas, through the self-contained HDF5 subset of h5file.cpp.
//
//   mesh file      src/mesh/mesh.cpp:16-26 (dataset names), 79-204 (read_mesh):
//                  Dimension, QOrder, nElem, nNode, nIFace, nNodePerElem,
//                  nNodePerFace (scalars), NodeCoords [nNode][dim],
//                  Elem2Nodes [nElem][nNodePerElem], IFaceData [nIFace][6] =
//                  (elemL, faceL, orientL, elemR, faceR, orientR), nBFaceGroup
//   solution file  src/io/writer.cpp:10-64 (Writer::write) with the parallel
//                  dataset convention of src/io/HDF5Wrapper.h:775-880: each
//                  per-rank array X is one 1-D dataset of the ranks' blocks
//                  back to back, X_offsets [nRanks] (attributes nDims, nRanks,
//                  totalSize) and X_dims [nRanks * nDims]; read back as
//                  Solver::read_in_coefficients (src/solver/base.cpp:234-279)
//                  and Reader (src/io/reader.h) do, both storage layouts.
#include <algorithm>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/dg_b200.h"
#include "h5file.h"

namespace dgi {
int fail(dg_ctx* c, int code, const std::string& msg);
}

namespace {

int ferr(int code, const std::string& msg) { return dgi::fail(nullptr, code, msg); }

bool scalar(h5::Reader& r, const char* name, int64_t& v, std::string& err)
{
    std::vector<int64_t> x;
    std::vector<uint64_t> dims;
    if (!r.read_int(name, x, &dims, err)) return false;
    if (x.size() != 1) {
        err = std::string(name) + " is not one value";
        return false;
    }
    v = x[0];
    return true;
}

// a parallel dataset (HDF5Wrapper.h:775-880): the blocks of all ranks, each
// with its dimensions
struct ParallelSet {
    std::vector<double> data;
    std::vector<int64_t> idata;
    std::vector<std::vector<uint64_t>> dims;  // per rank
    std::vector<uint64_t> offsets;            // per rank, in elements
};

bool read_parallel(h5::Reader& r, const std::string& name, bool integer, ParallelSet& s, std::string& err)
{
    int64_t nd = 0, nr = 0;
    std::vector<int64_t> offs, dall;
    if (!r.attr_int(name + "_offsets", "nDims", nd, err) || !r.attr_int(name + "_offsets", "nRanks", nr, err))
        return false;
    if (!r.read_int(name + "_offsets", offs, nullptr, err) || !r.read_int(name + "_dims", dall, nullptr, err)) return false;
    if (nd < 1 || nr < 1 || nd > 16 || nr > (1 << 24) || static_cast<int64_t>(offs.size()) != nr ||
        static_cast<int64_t>(dall.size()) != nd * nr) {
        err = name + ": inconsistent _offsets / _dims";
        return false;
    }
    uint64_t total = 0;
    if (integer) {
        if (!r.read_int(name, s.idata, nullptr, err)) return false;
        total = s.idata.size();
    } else {
        if (!r.read_double(name, s.data, nullptr, err)) return false;
        total = s.data.size();
    }
    s.dims.assign(nr, {});
    s.offsets.assign(nr, 0);
    for (int64_t k = 0; k < nr; ++k) {
        uint64_t n = 1;
        for (int64_t d = 0; d < nd; ++d) {
            const int64_t dk = dall[k * nd + d];
            if (dk < 0 || (dk > 0 && n > total / static_cast<uint64_t>(dk))) {
                err = name + ": rank block dimensions exceed the dataset";
                return false;
            }
            s.dims[k].push_back(static_cast<uint64_t>(dk));
            n *= s.dims[k].back();
        }
        if (offs[k] < 0 || static_cast<uint64_t>(offs[k]) + n > total) {
            err = name + ": rank block outside the dataset";
            return false;
        }
        s.offsets[k] = static_cast<uint64_t>(offs[k]);
    }
    return true;
}

// one parallel dataset of a single rank (Writer::write with one rank)
void write_parallel(h5::Writer& w, const std::string& name, const std::vector<uint64_t>& dims, h5::Type t,
                    const void* data)
{
    uint64_t total = 1;
    for (uint64_t d : dims) total *= d;
    w.dataset(name, {total}, t, data);
    const uint64_t zero = 0;
    w.dataset(name + "_offsets", {1}, h5::Type::u64(), &zero);
    const uint64_t nd = dims.size();
    const int32_t nranks = 1;
    w.attribute(name + "_offsets", "nDims", h5::Type::u64(), &nd);
    w.attribute(name + "_offsets", "nRanks", h5::Type::i32(), &nranks);
    w.attribute(name + "_offsets", "totalSize", h5::Type::u64(), &total);
    w.dataset(name + "_dims", {nd}, h5::Type::u64(), dims.data());
}

int dg_mesh_read_h5_impl(const char* path, int* dim, int* qorder, int* nnode_per_elem, int* nnode, double* node_coords,
                    int* nelem, unsigned* elem_to_node_ids, int* nface, unsigned* interior_faces)
{
    if (!path || !dim || !qorder || !nnode_per_elem || !nnode || !nelem || !nface)
        return ferr(DG_ERR_ARG, "dg_mesh_read_h5: null argument");
    h5::Reader r;
    std::string err;
    if (!r.open(path, err)) return ferr(DG_ERR_ARG, std::string("dg_mesh_read_h5: ") + err);
    int64_t d = 0, q = 0, ne = 0, nn = 0, nf = 0, npe = 0;
    if (!scalar(r, "Dimension", d, err) || !scalar(r, "QOrder", q, err) || !scalar(r, "nElem", ne, err) ||
        !scalar(r, "nNode", nn, err) || !scalar(r, "nIFace", nf, err) || !scalar(r, "nNodePerElem", npe, err))
        return ferr(DG_ERR_ARG, std::string("dg_mesh_read_h5: ") + path + ": " + err);
    if (d < 1 || d > 3 || q < 1 || ne < 1 || nn < 1 || nf < 0 || npe < 2 || ne > (1LL << 30) || nn > (1LL << 31) - 1 ||
        nf > (1LL << 31) - 1 || ne * npe > (1LL << 34))
        return ferr(DG_ERR_ARG, std::string("dg_mesh_read_h5: ") + path + ": sizes out of range");
    // the counts must be those of the stored arrays (a caller allocates from
    // them before the data is read)
    const std::pair<const char*, int64_t> stored[3] = {{"NodeCoords", nn * d}, {"Elem2Nodes", ne * npe},
                                                       {"IFaceData", nf * 6}};
    for (const auto& [name, want] : stored) {
        std::vector<uint64_t> dims;
        h5::Type ty;
        if (!r.shape(name, dims, ty, err)) return ferr(DG_ERR_ARG, std::string("dg_mesh_read_h5: ") + path + ": " + err);
        uint64_t total = 1;
        for (uint64_t n : dims) total = n > 0 && total > (1ULL << 62) / n ? 0 : total * n;
        if (total != static_cast<uint64_t>(want))
            return ferr(DG_ERR_ARG, std::string("dg_mesh_read_h5: ") + path + ": array sizes disagree with the counts");
    }
    *dim = static_cast<int>(d);
    *qorder = static_cast<int>(q);
    *nnode_per_elem = static_cast<int>(npe);
    *nnode = static_cast<int>(nn);
    *nelem = static_cast<int>(ne);
    *nface = static_cast<int>(nf);
    if (!node_coords && !elem_to_node_ids && !interior_faces) return DG_OK;
    if (!node_coords || !elem_to_node_ids || (nf > 0 && !interior_faces))
        return ferr(DG_ERR_ARG, "dg_mesh_read_h5: give all three arrays (or none for the sizes)");
    std::vector<double> xy;
    std::vector<int64_t> e2n, ifd;
    std::vector<uint64_t> dx, de, df;
    if (!r.read_double("NodeCoords", xy, &dx, err) || !r.read_int("Elem2Nodes", e2n, &de, err) ||
        !r.read_int("IFaceData", ifd, &df, err))
        return ferr(DG_ERR_ARG, std::string("dg_mesh_read_h5: ") + path + ": " + err);
    if (xy.size() != static_cast<size_t>(nn * d) || e2n.size() != static_cast<size_t>(ne * npe) ||
        ifd.size() != static_cast<size_t>(nf * 6))
        return ferr(DG_ERR_ARG, std::string("dg_mesh_read_h5: ") + path + ": array sizes disagree with the counts");
    for (int64_t v : e2n)
        if (v < 0 || v >= nn) return ferr(DG_ERR_ARG, "dg_mesh_read_h5: Elem2Nodes entry out of range");
    const int64_t nfaces_per_elem = 2 * d;
    for (int64_t f = 0; f < nf; ++f)
        for (int s = 0; s < 2; ++s) {
            const int64_t e = ifd[6 * f + 3 * s], lf = ifd[6 * f + 3 * s + 1], o = ifd[6 * f + 3 * s + 2];
            if (e < 0 || e >= ne || lf < 0 || lf >= nfaces_per_elem || o < 0 || o > 7)
                return ferr(DG_ERR_ARG, "dg_mesh_read_h5: IFaceData row " + std::to_string(f) + " out of range");
        }
    std::copy(xy.begin(), xy.end(), node_coords);
    for (size_t i = 0; i < e2n.size(); ++i) elem_to_node_ids[i] = static_cast<unsigned>(e2n[i]);
    // interior_faces rows (rankL, elemL, faceL, orientL, rankR, elemR, faceR, orientR), src/mesh/mesh.h:280-284
    for (int64_t f = 0; f < nf; ++f) {
        unsigned* row = interior_faces + 8 * f;
        for (int s = 0; s < 2; ++s) {
            row[4 * s] = 0;
            for (int k = 0; k < 3; ++k) row[4 * s + 1 + k] = static_cast<unsigned>(ifd[6 * f + 3 * s + k]);
        }
    }
    return DG_OK;
}

int dg_mesh_write_h5_impl(const char* path, const dg_mesh_desc* md)
{
    if (!path || !md || !md->node_coords || !md->elem_to_node_ids || (md->nface > 0 && !md->interior_faces) ||
        md->nnode < 1 || md->nelem < 1 || md->nface < 0)
        return ferr(DG_ERR_ARG, "dg_mesh_write_h5: bad argument");
    const int64_t ne = md->nelem, nn = md->nnode, nf = md->nface;
    std::vector<int64_t> e2n(ne * 8), ifd(nf * 6);
    for (int64_t i = 0; i < ne * 8; ++i) {
        if (md->elem_to_node_ids[i] >= static_cast<unsigned>(nn)) return ferr(DG_ERR_ARG, "dg_mesh_write_h5: node id out of range");
        e2n[i] = md->elem_to_node_ids[i];
    }
    for (int64_t f = 0; f < nf; ++f)
        for (int s = 0; s < 2; ++s)
            for (int k = 0; k < 3; ++k) ifd[6 * f + 3 * s + k] = md->interior_faces[8 * f + 4 * s + 1 + k];
    h5::Writer w;
    const int64_t three = 3, one = 1, eight = 8, four = 4, zero = 0;
    w.dataset("Dimension", {}, h5::Type::i64(), &three);
    w.dataset("QOrder", {}, h5::Type::i64(), &one);
    w.dataset("nElem", {}, h5::Type::i64(), &ne);
    w.dataset("nNode", {}, h5::Type::i64(), &nn);
    w.dataset("nIFace", {}, h5::Type::i64(), &nf);
    w.dataset("nNodePerElem", {}, h5::Type::i64(), &eight);
    w.dataset("nNodePerFace", {}, h5::Type::i64(), &four);
    w.dataset("nBFaceGroup", {}, h5::Type::i64(), &zero);
    w.dataset("NodeCoords", {static_cast<uint64_t>(nn), 3}, h5::Type::f64(), md->node_coords);
    w.dataset("Elem2Nodes", {static_cast<uint64_t>(ne), 8}, h5::Type::i64(), e2n.data());
    w.dataset("IFaceData", {static_cast<uint64_t>(nf), 6}, h5::Type::i64(), ifd.data());
    std::string err;
    if (!w.write(path, err)) return ferr(DG_ERR_ARG, "dg_mesh_write_h5: " + err);
    return DG_OK;
}

// Writer::write for one rank: dim-D mesh of npe-node elements, ns variables
int solution_write(const char* fn, const char* path, int dim, int npe, int ns, int nnode, const double* coords,
                   int nelem, const unsigned* e2n_in, int nb, const double* Uc, double time)
{
    const uint64_t ne = nelem, nn = nnode;
    h5::Writer w;
    const uint32_t u_ranks = 1, u_dim = static_cast<uint32_t>(dim), u_ne = static_cast<uint32_t>(ne),
                   u_nn = static_cast<uint32_t>(nn), u_npe = static_cast<uint32_t>(npe), u_nb = static_cast<uint32_t>(nb),
                   u_ns = static_cast<uint32_t>(ns);
    const int32_t row_major = 1;  // "Stored Layout": LayoutRight, written as an int (HDF5Wrapper.h:212-215)
    w.attribute("", "Number of Ranks", h5::Type::u32(), &u_ranks);
    w.attribute("", "Number of Dimensions", h5::Type::u32(), &u_dim);
    w.attribute("", "Number of Elements", h5::Type::u32(), &u_ne);
    w.attribute("", "Number of Nodes", h5::Type::u32(), &u_nn);
    w.attribute("", "Number of Nodes Per Element", h5::Type::u32(), &u_npe);
    w.attribute("", "Number of Basis Functions", h5::Type::u32(), &u_nb);
    w.attribute("", "Number of State Variables", h5::Type::u32(), &u_ns);
    w.attribute("", "Solver Final Time", h5::Type::f64(), &time);
    w.attribute("", "Stored Layout", h5::Type::i32(), &row_major);
    w.dataset("Number of Elements per Partition", {1}, h5::Type::u32(), &u_ne);
    std::vector<uint32_t> l2g_node(nn), l2g_elem(ne), e2n(ne * npe);
    for (uint64_t i = 0; i < nn; ++i) l2g_node[i] = static_cast<uint32_t>(i);
    for (uint64_t i = 0; i < ne; ++i) l2g_elem[i] = static_cast<uint32_t>(i);
    for (uint64_t i = 0; i < ne * npe; ++i) e2n[i] = e2n_in[i];
    write_parallel(w, "Node Coordinates", {nn, static_cast<uint64_t>(dim)}, h5::Type::f64(), coords);
    write_parallel(w, "Local to Global Node ID", {nn}, h5::Type::u32(), l2g_node.data());
    write_parallel(w, "Element Global Node IDs", {ne, static_cast<uint64_t>(npe)}, h5::Type::u32(), e2n.data());
    write_parallel(w, "Local to Global Element IDs", {ne}, h5::Type::u32(), l2g_elem.data());
    write_parallel(w, "Solution Coefficients", {ne, static_cast<uint64_t>(nb), static_cast<uint64_t>(ns)}, h5::Type::f64(), Uc);
    std::string err;
    if (!w.write(path, err)) return ferr(DG_ERR_ARG, std::string(fn) + ": " + err);
    return DG_OK;
}

int dg_solution_write_h5_impl(const char* path, const dg_mesh_desc* md, int order, const double* Uc, double time)
{
    if (!path || !md || !md->node_coords || !md->elem_to_node_ids || !Uc || md->nnode < 1 || md->nelem < 1 ||
        order < 0 || order > 5)
        return ferr(DG_ERR_ARG, "dg_solution_write_h5: bad argument");
    const int nb = (order + 1) * (order + 1) * (order + 1);
    return solution_write("dg_solution_write_h5", path, 3, 8, 5, md->nnode, md->node_coords, md->nelem,
                          md->elem_to_node_ids, nb, Uc, time);
}

int dg2d_solution_write_h5_impl(const char* path, const dg_mesh2d_desc* md, int order, const double* Uc, double time)
{
    if (!path || !md || !md->node_coords || !md->elem_to_node_ids || !Uc || md->nnode < 1 || md->nelem < 1 ||
        order < 0 || order > 5)
        return ferr(DG_ERR_ARG, "dg2d_solution_write_h5: bad argument");
    const int nb = (order + 1) * (order + 1);
    return solution_write("dg2d_solution_write_h5", path, 2, 4, 4, md->nnode, md->node_coords, md->nelem,
                          md->elem_to_node_ids, nb, Uc, time);
}

int dg_solution_read_h5_impl(const char* path, int* nelem, int* nb, int* ns, double* time, double* Uc)
{
    if (!path || !nelem || !nb || !ns || !time) return ferr(DG_ERR_ARG, "dg_solution_read_h5: null argument");
    h5::Reader r;
    std::string err;
    if (!r.open(path, err)) return ferr(DG_ERR_ARG, std::string("dg_solution_read_h5: ") + err);
    int64_t ne = 0, b = 0, s = 0, layout = 1;
    double t = 0.0;
    if (!r.attr_int("", "Number of Elements", ne, err) || !r.attr_int("", "Number of Basis Functions", b, err) ||
        !r.attr_int("", "Number of State Variables", s, err) || !r.attr_double("", "Solver Final Time", t, err) ||
        !r.attr_int("", "Stored Layout", layout, err))
        return ferr(DG_ERR_ARG, std::string("dg_solution_read_h5: ") + path + ": " + err);
    if (ne < 1 || b < 1 || s < 1 || ne > (1LL << 30) || b > 4096 || s > 64)
        return ferr(DG_ERR_ARG, "dg_solution_read_h5: sizes out of range");
    // the sizes must be those of the stored coefficients (a caller allocates
    // from them before the data is read)
    {
        std::vector<uint64_t> dims;
        h5::Type ty;
        if (!r.shape("Solution Coefficients", dims, ty, err))
            return ferr(DG_ERR_ARG, std::string("dg_solution_read_h5: ") + path + ": " + err);
        uint64_t total = 1;
        for (uint64_t d : dims) total = d > 0 && total > (1ULL << 62) / d ? 0 : total * d;
        if (dims.empty() || total != static_cast<uint64_t>(ne) * static_cast<uint64_t>(b) * static_cast<uint64_t>(s))
            return ferr(DG_ERR_ARG, "dg_solution_read_h5: element, basis and variable counts disagree with the stored coefficients");
    }
    *nelem = static_cast<int>(ne);
    *nb = static_cast<int>(b);
    *ns = static_cast<int>(s);
    *time = t;
    if (!Uc) return DG_OK;
    ParallelSet U, ids;
    if (!read_parallel(r, "Solution Coefficients", false, U, err) ||
        !read_parallel(r, "Local to Global Element IDs", true, ids, err))
        return ferr(DG_ERR_ARG, std::string("dg_solution_read_h5: ") + path + ": " + err);
    if (U.dims.size() != ids.dims.size()) return ferr(DG_ERR_ARG, "dg_solution_read_h5: rank counts disagree");
    // every rank's block of elements to its global element ids (Reader's
    // serialisation, src/io/reader.h:60-80), in either storage layout
    // (read_in_coefficients, src/solver/base.cpp:257-274)
    std::vector<char> seen(ne, 0);
    const uint64_t per = static_cast<uint64_t>(b * s);
    for (size_t k = 0; k < U.dims.size(); ++k) {
        const std::vector<uint64_t>& d = U.dims[k];
        if (d.size() != 3 || d[1] != static_cast<uint64_t>(b) || d[2] != static_cast<uint64_t>(s) ||
            ids.dims[k].size() != 1 || ids.dims[k][0] != d[0])
            return ferr(DG_ERR_ARG, "dg_solution_read_h5: rank block dimensions disagree");
        const uint64_t nek = d[0];
        const double* blk = U.data.data() + U.offsets[k];
        for (uint64_t i = 0; i < nek; ++i) {
            const int64_t g = ids.idata[ids.offsets[k] + i];
            if (g < 0 || g >= ne || seen[g]) return ferr(DG_ERR_ARG, "dg_solution_read_h5: element ids are not a permutation");
            seen[g] = 1;
            double* dst = Uc + static_cast<uint64_t>(g) * per;
            for (int64_t j = 0; j < b; ++j)
                for (int64_t v = 0; v < s; ++v)
                    dst[j * s + v] = layout ? blk[i * per + j * s + v] : blk[(v * b + j) * nek + i];
        }
    }
    if (std::find(seen.begin(), seen.end(), 0) != seen.end())
        return ferr(DG_ERR_ARG, "dg_solution_read_h5: the file does not hold every element");
    return DG_OK;
}

// the C ABI: no exception crosses it (an allocation a corrupt file asks for
// becomes DG_ERR_NOMEM)
template <typename F>
int guarded(const char* fn, F&& f)
{
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return ferr(DG_ERR_NOMEM, std::string(fn) + ": out of host memory");
    } catch (const std::exception& e) {
        return ferr(DG_ERR_ARG, std::string(fn) + ": " + e.what());
    }
}

}  // namespace

extern "C" {

int dg_mesh_read_h5(const char* path, int* dim, int* qorder, int* nnode_per_elem, int* nnode, double* node_coords,
                    int* nelem, unsigned* elem_to_node_ids, int* nface, unsigned* interior_faces)
{
    return guarded("dg_mesh_read_h5", [&] {
        return dg_mesh_read_h5_impl(path, dim, qorder, nnode_per_elem, nnode, node_coords, nelem, elem_to_node_ids,
                                    nface, interior_faces);
    });
}

int dg_mesh_write_h5(const char* path, const dg_mesh_desc* md)
{
    return guarded("dg_mesh_write_h5", [&] { return dg_mesh_write_h5_impl(path, md); });
}

int dg_solution_write_h5(const char* path, const dg_mesh_desc* md, int order, const double* Uc, double time)
{
    return guarded("dg_solution_write_h5", [&] { return dg_solution_write_h5_impl(path, md, order, Uc, time); });
}

int dg_solution_read_h5(const char* path, int* nelem, int* nb, int* ns, double* time, double* Uc)
{
    return guarded("dg_solution_read_h5", [&] { return dg_solution_read_h5_impl(path, nelem, nb, ns, time, Uc); });
}

int dg2d_solution_write_h5(const char* path, const dg_mesh2d_desc* md, int order, const double* Uc, double time)
{
    return guarded("dg2d_solution_write_h5", [&] { return dg2d_solution_write_h5_impl(path, md, order, Uc, time); });
}

}  // extern "C"
