// h5file.h -- a self-contained reader and writer for the subset of the HDF5
// file format that the reference's mesh and solution files use, so that the
// drop-in reads the reference's meshes (src/mesh/mesh.cpp:79-204) and writes
// data.h5 in the reference writer's schema (src/io/writer.cpp:10-64,
// src/io/HDF5Wrapper.h:347-880) without the HDF5 library, which this build
// does not link.
//
// The subset (HDF5 File Format Specification, version 0 superblock family):
//   superblock version 0 or 1, 8-byte offsets and lengths, little endian;
//   groups as symbol tables (version 1 B-tree of symbol nodes + local heap) or
//   as link messages (hard links, compact storage); version 1 object headers
//   with continuation blocks; dataspaces (scalar or simple), fixed-point and
//   IEEE floating-point datatypes; contiguous and compact data layouts
//   (layout message version 3); attribute messages versions 1-3.
// Anything else (version 2/3 superblocks and object headers, chunked or
// filtered datasets, dense link storage, big-endian or compound types) is
// reported as unsupported, never guessed.
//
// The writer emits exactly this subset: a version 0 superblock, a root group
// stored as a symbol table (one B-tree leaf over symbol nodes of at most
// 2 * 4 entries, the default leaf K), datasets with version 1 object headers
// and contiguous layout, attributes as version 1 attribute messages.  Only
// objects in the root group, as both schemas use.
#pragma once
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace h5 {

// element type of a dataset or attribute
struct Type {
    int cls = -1;          // 0 fixed-point (integer), 1 IEEE floating point
    int size = 0;          // bytes
    bool is_signed = false;
    static Type i32() { return {0, 4, true}; }
    static Type u32() { return {0, 4, false}; }
    static Type i64() { return {0, 8, true}; }
    static Type u64() { return {0, 8, false}; }
    static Type f64() { return {1, 8, true}; }
};

class Reader {
public:
    Reader() = default;
    ~Reader();
    Reader(const Reader&) = delete;
    Reader& operator=(const Reader&) = delete;

    // opens the file and reads the root group's links; false with err set on failure
    bool open(const std::string& path, std::string& err);
    // names of the root group's links, in the group's order
    const std::vector<std::string>& names() const { return names_; }
    bool has(const std::string& name) const;

    // a root-group dataset's shape and element type
    bool shape(const std::string& name, std::vector<uint64_t>& dims, Type& type, std::string& err);
    // a root-group dataset's elements converted to int64 / double (integer
    // datasets read as double only if every value is exact)
    bool read_int(const std::string& name, std::vector<int64_t>& out, std::vector<uint64_t>* dims, std::string& err);
    bool read_double(const std::string& name, std::vector<double>& out, std::vector<uint64_t>* dims, std::string& err);
    // a scalar (or one-element) attribute of the root group (obj = "") or of a
    // root-group dataset
    bool attr_int(const std::string& obj, const std::string& name, int64_t& v, std::string& err);
    bool attr_double(const std::string& obj, const std::string& name, double& v, std::string& err);
    bool has_attr(const std::string& obj, const std::string& name);

private:
    struct Msg {
        int type;
        std::vector<uint8_t> data;
    };
    struct Dset {
        std::vector<uint64_t> dims;
        Type type;
        int layout = -1;   // 0 compact, 1 contiguous
        uint64_t addr = 0, bytes = 0;
        std::vector<uint8_t> compact;
    };
    struct Attr {
        std::string name;
        std::vector<uint64_t> dims;
        Type type;
        std::vector<uint8_t> data;
    };
    bool rd(uint64_t addr, void* dst, uint64_t n, std::string& err);
    bool header(uint64_t addr, std::vector<Msg>& msgs, std::string& err);
    bool group_btree(uint64_t btree, const std::vector<uint8_t>& heap, int level_expected, long& budget,
                     std::string& err);
    bool heap_data(uint64_t addr, std::vector<uint8_t>& data, std::string& err);
    bool object(const std::string& name, uint64_t& addr, std::string& err) const;
    bool dataset(const std::string& name, Dset& d, std::string& err);
    bool attributes(const std::string& obj, std::vector<Attr>& out, std::string& err);
    bool payload(const Dset& d, std::vector<uint8_t>& raw, std::string& err);

    FILE* f_ = nullptr;
    uint64_t base_ = 0, eof_ = 0, root_ = 0;
    std::vector<std::string> names_;
    std::vector<uint64_t> addrs_;
};

class Writer {
public:
    // a dataset of the root group; data holds prod(dims) elements of `type`
    // (copied); an empty dims makes a scalar dataset
    void dataset(const std::string& name, const std::vector<uint64_t>& dims, Type type, const void* data);
    // a scalar attribute of the root group (obj = "") or of a dataset added
    // before (value: one element of `type`)
    void attribute(const std::string& obj, const std::string& name, Type type, const void* value);
    // writes the file; false with err set on failure (names must be unique,
    // non-empty and free of '/')
    bool write(const std::string& path, std::string& err) const;

private:
    struct A {
        std::string name;
        Type type;
        std::vector<uint8_t> value;
    };
    struct D {
        std::string name;
        std::vector<uint64_t> dims;
        Type type;
        std::vector<uint8_t> data;
        std::vector<A> attrs;
    };
    std::vector<D> dsets_;
    std::vector<A> root_attrs_;
};

}  // namespace h5
