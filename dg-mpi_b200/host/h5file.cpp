// h5file.cpp -- the HDF5 subset reader and writer (see h5file.h).
#include "h5file.h"

#include <algorithm>
#include <cstring>

namespace h5 {

namespace {

constexpr uint64_t kUndef = ~0ull;
constexpr uint8_t kSig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
constexpr int kLeafK = 4;        // symbol-node capacity 2K (the format's default)
constexpr int kInternalK = 16;   // B-tree node capacity 2K (the format's default)
constexpr uint64_t kBtreeBytes = 24 + 2 * kInternalK * 8 + (2 * kInternalK + 1) * 8;
constexpr uint64_t kSnodBytes = 8 + 2 * kLeafK * 40;

// message types of version 1 object headers
enum : int {
    kMsgNil = 0x00, kMsgDataspace = 0x01, kMsgLinkInfo = 0x02, kMsgDatatype = 0x03, kMsgFillOld = 0x04,
    kMsgFill = 0x05, kMsgLink = 0x06, kMsgLayout = 0x08, kMsgFilters = 0x0B, kMsgAttribute = 0x0C,
    kMsgContinuation = 0x10, kMsgSymbolTable = 0x11,
};

uint64_t le(const uint8_t* p, int n)
{
    uint64_t v = 0;
    for (int i = n - 1; i >= 0; --i) v = (v << 8) | p[i];
    return v;
}

uint64_t pad8(uint64_t n) { return (n + 7) & ~7ull; }

uint64_t count(const std::vector<uint64_t>& dims)
{
    uint64_t n = 1;
    for (uint64_t d : dims) n *= d;
    return n;
}

// the element count, or false if it (times an element size of up to 16
// bytes) does not fit in 2^60
bool count_ok(const std::vector<uint64_t>& dims, uint64_t& n)
{
    n = 1;
    for (uint64_t d : dims) {
        if (d != 0 && n > (1ull << 56) / d) return false;
        n *= d;
    }
    return true;
}

// dataspace message (versions 1 and 2): rank and current dimensions
bool decode_dataspace(const uint8_t* p, size_t n, std::vector<uint64_t>& dims, std::string& err)
{
    if (n < 4) { err = "short dataspace message"; return false; }
    const int ver = p[0], rank = p[1];
    size_t off;
    if (ver == 1) off = 8;
    else if (ver == 2) {
        if (p[3] == 2) { err = "null dataspace"; return false; }
        off = 4;
    } else { err = "dataspace message version " + std::to_string(ver); return false; }
    if (n < off + 8ull * rank) { err = "short dataspace message"; return false; }
    dims.resize(rank);
    for (int i = 0; i < rank; ++i) dims[i] = le(p + off + 8 * i, 8);
    return true;
}

// datatype message: little-endian integers and IEEE binary32/binary64 only
bool decode_datatype(const uint8_t* p, size_t n, Type& t, std::string& err)
{
    if (n < 8) { err = "short datatype message"; return false; }
    const int cls = p[0] & 15;
    const uint8_t b1 = p[1];
    t.size = static_cast<int>(le(p + 4, 4));
    if (cls == 0) {
        if (n < 12) { err = "short datatype message"; return false; }
        if (b1 & 1) { err = "big-endian integer type"; return false; }
        const int prec = static_cast<int>(le(p + 10, 2));
        if (le(p + 8, 2) != 0 || prec != 8 * t.size || (t.size != 1 && t.size != 2 && t.size != 4 && t.size != 8)) {
            err = "integer type with padding bits";
            return false;
        }
        t.cls = 0;
        t.is_signed = (b1 >> 3) & 1;
        return true;
    }
    if (cls == 1) {
        if (n < 20) { err = "short datatype message"; return false; }
        if ((b1 & 1) || ((b1 >> 6) & 1)) { err = "non-little-endian floating-point type"; return false; }
        const int prec = static_cast<int>(le(p + 10, 2)), eloc = p[12], esz = p[13], mloc = p[14], msz = p[15];
        const uint64_t bias = le(p + 16, 4);
        const bool f64 = t.size == 8 && prec == 64 && eloc == 52 && esz == 11 && mloc == 0 && msz == 52 && bias == 1023;
        const bool f32 = t.size == 4 && prec == 32 && eloc == 23 && esz == 8 && mloc == 0 && msz == 23 && bias == 127;
        if (!(f64 || f32) || le(p + 8, 2) != 0 || ((b1 >> 4) & 3) != 2 || p[2] != 8 * t.size - 1) {
            err = "floating-point type other than IEEE binary32/binary64";
            return false;
        }
        t.cls = 1;
        t.is_signed = true;
        return true;
    }
    err = "datatype class " + std::to_string(cls) + " (only integer and floating point are read)";
    return false;
}

// element i of a raw buffer of type t, as int64 / double
int64_t elem_int(const uint8_t* raw, const Type& t, uint64_t i)
{
    const uint64_t u = le(raw + i * t.size, t.size);
    if (!t.is_signed || t.size == 8) return static_cast<int64_t>(u);
    const uint64_t sign = 1ull << (8 * t.size - 1);
    return static_cast<int64_t>((u ^ sign) - sign);
}
double elem_double(const uint8_t* raw, const Type& t, uint64_t i)
{
    if (t.size == 8) {
        double d;
        std::memcpy(&d, raw + i * 8, 8);
        return d;
    }
    float f;
    std::memcpy(&f, raw + i * 4, 4);
    return f;
}

// ---- writer encoding ----
struct Buf {
    std::vector<uint8_t> b;
    void u8(uint64_t v) { b.push_back(static_cast<uint8_t>(v)); }
    void u(uint64_t v, int n)
    {
        for (int i = 0; i < n; ++i) b.push_back(static_cast<uint8_t>(v >> (8 * i)));
    }
    void raw(const void* p, size_t n)
    {
        const uint8_t* c = static_cast<const uint8_t*>(p);
        b.insert(b.end(), c, c + n);
    }
    void align8() { b.resize(pad8(b.size()), 0); }
    size_t size() const { return b.size(); }
};

std::vector<uint8_t> enc_datatype(const Type& t)
{
    Buf m;
    if (t.cls == 0) {
        m.u8(0x10);
        m.u8(t.is_signed ? 0x08 : 0x00);
        m.u8(0);
        m.u8(0);
        m.u(t.size, 4);
        m.u(0, 2);
        m.u(8 * t.size, 2);
    } else {
        m.u8(0x11);
        m.u8(0x20);                 // mantissa normalisation: implied leading bit
        m.u8(8 * t.size - 1);       // sign bit position
        m.u8(0);
        m.u(t.size, 4);
        m.u(0, 2);
        m.u(8 * t.size, 2);
        m.u8(t.size == 8 ? 52 : 23);  // exponent position
        m.u8(t.size == 8 ? 11 : 8);   // exponent bits
        m.u8(0);                      // mantissa position
        m.u8(t.size == 8 ? 52 : 23);  // mantissa bits
        m.u(t.size == 8 ? 1023 : 127, 4);
    }
    return m.b;
}

std::vector<uint8_t> enc_dataspace(const std::vector<uint64_t>& dims)
{
    Buf m;
    m.u8(1);
    m.u8(dims.size());
    m.u8(dims.empty() ? 0 : 1);  // maximum dimensions present (equal to the current ones)
    m.u8(0);
    m.u(0, 4);
    for (uint64_t d : dims) m.u(d, 8);
    for (uint64_t d : dims) m.u(d, 8);
    return m.b;
}

std::vector<uint8_t> enc_attribute(const std::string& name, const Type& t, const std::vector<uint8_t>& value)
{
    const std::vector<uint8_t> dt = enc_datatype(t), ds = enc_dataspace({});
    Buf m;
    m.u8(1);
    m.u8(0);
    m.u(name.size() + 1, 2);
    m.u(dt.size(), 2);
    m.u(ds.size(), 2);
    m.raw(name.c_str(), name.size() + 1);
    m.align8();
    m.raw(dt.data(), dt.size());
    m.align8();
    m.raw(ds.data(), ds.size());
    m.align8();
    m.raw(value.data(), value.size());
    return m.b;
}

struct HMsg {
    int type;
    std::vector<uint8_t> data;
    int flags = 0;  // 1: constant (datatype and fill value messages, as the library marks them)
};

// a version 1 object header holding `msgs`
std::vector<uint8_t> enc_header(const std::vector<HMsg>& msgs)
{
    Buf body;
    for (const HMsg& m : msgs) {
        body.u(m.type, 2);
        body.u(pad8(m.data.size()), 2);
        body.u8(m.flags);
        body.u(0, 3);
        body.raw(m.data.data(), m.data.size());
        body.align8();
    }
    Buf h;
    h.u8(1);
    h.u8(0);
    h.u(msgs.size(), 2);
    h.u(1, 4);  // reference count
    h.u(body.size(), 4);
    h.u(0, 4);  // alignment of the first message to 8 bytes
    h.raw(body.b.data(), body.size());
    return h.b;
}

}  // namespace

// ======================= Reader =======================

Reader::~Reader()
{
    if (f_) std::fclose(f_);
}

bool Reader::rd(uint64_t addr, void* dst, uint64_t n, std::string& err)
{
    if (addr == kUndef || base_ + addr + n > eof_ || base_ + addr + n < base_ + addr) {
        err = "address out of the file";
        return false;
    }
    if (fseeko(f_, static_cast<off_t>(base_ + addr), SEEK_SET) != 0 || std::fread(dst, 1, n, f_) != n) {
        err = "read failed";
        return false;
    }
    return true;
}

bool Reader::header(uint64_t addr, std::vector<Msg>& msgs, std::string& err)
{
    uint8_t pre[16];
    if (!rd(addr, pre, 16, err)) return false;
    if (std::memcmp(pre, "OHDR", 4) == 0) {
        err = "version 2 object header (files written for the latest format versions are not read)";
        return false;
    }
    if (pre[0] != 1) {
        err = "object header version " + std::to_string(pre[0]);
        return false;
    }
    const uint64_t nmsg = le(pre + 2, 2);
    std::vector<std::pair<uint64_t, uint64_t>> blocks{{addr + 16, le(pre + 8, 4)}};
    msgs.clear();
    for (size_t b = 0; b < blocks.size() && b < 4096; ++b) {
        if (blocks[b].second > eof_) { err = "object header block larger than the file"; return false; }
        std::vector<uint8_t> blk(blocks[b].second);
        if (!rd(blocks[b].first, blk.data(), blk.size(), err)) return false;
        size_t pos = 0;
        while (pos + 8 <= blk.size() && msgs.size() < nmsg) {
            const int type = static_cast<int>(le(&blk[pos], 2));
            const size_t sz = le(&blk[pos + 2], 2);
            const uint8_t flags = blk[pos + 4];
            if (pos + 8 + sz > blk.size()) {
                err = "object header message runs past its block";
                return false;
            }
            if ((flags & 2) && type != kMsgNil) {
                err = "shared object header message";
                return false;
            }
            Msg m{type, std::vector<uint8_t>(blk.begin() + pos + 8, blk.begin() + pos + 8 + sz)};
            if (type == kMsgContinuation) {
                if (sz < 16) { err = "short continuation message"; return false; }
                blocks.push_back({le(m.data.data(), 8), le(m.data.data() + 8, 8)});
            }
            msgs.push_back(std::move(m));
            pos += 8 + sz;
        }
    }
    return true;
}

bool Reader::heap_data(uint64_t addr, std::vector<uint8_t>& data, std::string& err)
{
    uint8_t h[32];
    if (!rd(addr, h, 32, err)) return false;
    if (std::memcmp(h, "HEAP", 4) != 0 || h[4] != 0) {
        err = "bad local heap";
        return false;
    }
    const uint64_t n = le(h + 8, 8);
    if (n > eof_) { err = "local heap larger than the file"; return false; }
    data.resize(n);
    return rd(le(h + 24, 8), data.data(), data.size(), err);
}

bool Reader::group_btree(uint64_t btree, const std::vector<uint8_t>& heap, int level_expected, long& budget,
                         std::string& err)
{
    // every node is visited at most once per budget unit, and a child sits one
    // level below its parent: a corrupt tree (a cycle, a node shared by many
    // parents) ends in an error instead of an endless or exponential walk
    if (--budget < 0) { err = "group B-tree has too many nodes"; return false; }
    uint8_t h[24];
    if (!rd(btree, h, 24, err)) return false;
    if (std::memcmp(h, "TREE", 4) != 0 || h[4] != 0) {
        err = "bad group B-tree node";
        return false;
    }
    const int level = h[5];
    if (level_expected >= 0 && level != level_expected) {
        err = "group B-tree child is not one level below its parent";
        return false;
    }
    const uint64_t used = le(h + 6, 2);
    std::vector<uint8_t> kc(8 + 16 * used);
    if (!rd(btree + 24, kc.data(), kc.size(), err)) return false;
    for (uint64_t i = 0; i < used; ++i) {
        const uint64_t child = le(&kc[8 + 16 * i], 8);
        if (level > 0) {
            if (!group_btree(child, heap, level - 1, budget, err)) return false;
            continue;
        }
        uint8_t s[8];
        if (!rd(child, s, 8, err)) return false;
        if (std::memcmp(s, "SNOD", 4) != 0 || s[4] != 1) {
            err = "bad symbol table node";
            return false;
        }
        const uint64_t nsym = le(s + 6, 2);
        std::vector<uint8_t> ent(40 * nsym);
        if (!rd(child + 8, ent.data(), ent.size(), err)) return false;
        for (uint64_t k = 0; k < nsym; ++k) {
            const uint64_t off = le(&ent[40 * k], 8);
            if (off >= heap.size()) { err = "symbol name outside the local heap"; return false; }
            const char* c = reinterpret_cast<const char*>(heap.data() + off);
            names_.emplace_back(c, strnlen(c, heap.size() - off));
            addrs_.push_back(le(&ent[40 * k + 8], 8));
        }
    }
    return true;
}

bool Reader::open(const std::string& path, std::string& err)
{
    if (f_) { std::fclose(f_); f_ = nullptr; }
    names_.clear();
    addrs_.clear();
    f_ = std::fopen(path.c_str(), "rb");
    if (!f_) { err = "cannot open " + path; return false; }
    fseeko(f_, 0, SEEK_END);
    const uint64_t size = static_cast<uint64_t>(ftello(f_));
    eof_ = size;
    // the signature sits at 0, 512, 1024, 2048, ... (after a user block)
    uint64_t at = kUndef;
    for (uint64_t o = 0; o + 96 <= size; o = o ? 2 * o : 512) {
        uint8_t s[8];
        base_ = 0;
        if (!rd(o, s, 8, err)) return false;
        if (std::memcmp(s, kSig, 8) == 0) { at = o; break; }
    }
    if (at == kUndef) { err = path + " is not an HDF5 file"; return false; }
    uint8_t sb[100];
    if (!rd(at, sb, 24, err)) return false;
    const int ver = sb[8];
    if (ver > 1) {
        err = "superblock version " + std::to_string(ver) + " (files written for the latest format versions are not read)";
        return false;
    }
    if (sb[13] != 8 || sb[14] != 8) { err = "offsets or lengths other than 8 bytes"; return false; }
    const uint64_t vars = at + 24 + (ver == 1 ? 4 : 0);
    if (!rd(vars, sb, 72, err)) return false;
    base_ = le(sb, 8);
    // addresses are relative to the base address; the end-of-file address bounds reads
    const uint64_t eof_rel = le(sb + 16, 8);
    eof_ = std::min<uint64_t>(size, base_ + eof_rel);
    root_ = le(sb + 32 + 8, 8);
    std::vector<Msg> msgs;
    if (!header(root_, msgs, err)) return false;
    bool found = false;
    for (const Msg& m : msgs) {
        if (m.type == kMsgSymbolTable) {
            if (m.data.size() < 16) { err = "short symbol table message"; return false; }
            std::vector<uint8_t> heap;
            if (!heap_data(le(m.data.data() + 8, 8), heap, err)) return false;
            long budget = 1 << 16;
            if (!group_btree(le(m.data.data(), 8), heap, -1, budget, err)) return false;
            found = true;
        } else if (m.type == kMsgLinkInfo) {
            if (m.data.size() >= 10 && le(m.data.data() + 2 + ((m.data[1] & 1) ? 8 : 0), 8) != kUndef) {
                err = "group with dense link storage";
                return false;
            }
        } else if (m.type == kMsgLink) {
            // version 1 link message: hard links only
            const uint8_t* p = m.data.data();
            const size_t n = m.data.size();
            if (n < 2 || p[0] != 1) { err = "link message version"; return false; }
            const uint8_t fl = p[1];
            size_t pos = 2;
            int ltype = 0;
            if (fl & 8) {
                if (pos >= n) { err = "short link message"; return false; }
                ltype = p[pos++];
            }
            if (fl & 4) pos += 8;
            if (fl & 16) pos += 1;
            const int lsz = 1 << (fl & 3);
            if (pos + lsz > n) { err = "short link message"; return false; }
            const uint64_t nlen = le(p + pos, lsz);
            pos += lsz;
            if (ltype != 0) { err = "soft or external link"; return false; }
            if (nlen > n || pos + nlen + 8 > n) { err = "short link message"; return false; }
            names_.emplace_back(reinterpret_cast<const char*>(p + pos), nlen);
            addrs_.push_back(le(p + pos + nlen, 8));
            found = true;
        }
    }
    if (!found && names_.empty()) {
        // an empty group written with link messages has none; a symbol table is required otherwise
        bool has_links = false;
        for (const Msg& m : msgs) has_links |= m.type == kMsgLinkInfo;
        if (!has_links) { err = "root object is not a group"; return false; }
    }
    return true;
}

bool Reader::has(const std::string& name) const
{
    return std::find(names_.begin(), names_.end(), name) != names_.end();
}

bool Reader::object(const std::string& name, uint64_t& addr, std::string& err) const
{
    if (name.empty()) { addr = root_; return true; }
    for (size_t i = 0; i < names_.size(); ++i)
        if (names_[i] == name) { addr = addrs_[i]; return true; }
    err = "no object named '" + name + "'";
    return false;
}

bool Reader::dataset(const std::string& name, Dset& d, std::string& err)
{
    uint64_t addr;
    if (!object(name, addr, err)) return false;
    std::vector<Msg> msgs;
    if (!header(addr, msgs, err)) return false;
    bool space = false, type = false;
    for (const Msg& m : msgs) {
        const uint8_t* p = m.data.data();
        const size_t n = m.data.size();
        switch (m.type) {
            case kMsgDataspace: if (!decode_dataspace(p, n, d.dims, err)) return false; space = true; break;
            case kMsgDatatype: if (!decode_datatype(p, n, d.type, err)) return false; type = true; break;
            case kMsgFilters: err = "filtered dataset"; return false;
            case kMsgLayout:
                if (n < 2 || p[0] != 3) { err = "data layout message version " + std::to_string(n ? p[0] : 0); return false; }
                if (p[1] == 0) {
                    if (n < 4) { err = "short layout message"; return false; }
                    const uint64_t sz = le(p + 2, 2);
                    if (n < 4 + sz) { err = "short compact data"; return false; }
                    d.layout = 0;
                    d.compact.assign(p + 4, p + 4 + sz);
                } else if (p[1] == 1) {
                    if (n < 18) { err = "short layout message"; return false; }
                    d.layout = 1;
                    d.addr = le(p + 2, 8);
                    d.bytes = le(p + 10, 8);
                } else {
                    err = "chunked or virtual dataset layout";
                    return false;
                }
                break;
            default: break;
        }
    }
    if (!space || !type || d.layout < 0) {
        err = "'" + name + "' is not a dataset";
        return false;
    }
    return true;
}

bool Reader::payload(const Dset& d, std::vector<uint8_t>& raw, std::string& err)
{
    uint64_t n;
    if (!count_ok(d.dims, n)) { err = "dataspace too large"; return false; }
    const uint64_t bytes = n * d.type.size;
    if (d.layout == 1 && d.addr != kUndef && bytes > eof_) { err = "dataset larger than the file"; return false; }
    if (d.layout == 1 && d.addr == kUndef && bytes > (1ull << 34)) { err = "unallocated dataset too large"; return false; }
    raw.assign(bytes, 0);
    if (d.layout == 0) {
        if (d.compact.size() < bytes) { err = "short compact data"; return false; }
        std::memcpy(raw.data(), d.compact.data(), bytes);
        return true;
    }
    if (d.addr == kUndef) return true;  // never written: the fill value, zero
    if (d.bytes < bytes) { err = "contiguous storage smaller than the dataspace"; return false; }
    return bytes == 0 || rd(d.addr, raw.data(), bytes, err);
}

bool Reader::shape(const std::string& name, std::vector<uint64_t>& dims, Type& type, std::string& err)
{
    Dset d;
    if (!dataset(name, d, err)) return false;
    dims = d.dims;
    type = d.type;
    return true;
}

bool Reader::read_int(const std::string& name, std::vector<int64_t>& out, std::vector<uint64_t>* dims, std::string& err)
{
    Dset d;
    std::vector<uint8_t> raw;
    if (!dataset(name, d, err) || !payload(d, raw, err)) return false;
    if (d.type.cls != 0) { err = "'" + name + "' is not an integer dataset"; return false; }
    const uint64_t n = count(d.dims);
    out.resize(n);
    for (uint64_t i = 0; i < n; ++i) out[i] = elem_int(raw.data(), d.type, i);
    if (dims) *dims = d.dims;
    return true;
}

bool Reader::read_double(const std::string& name, std::vector<double>& out, std::vector<uint64_t>* dims, std::string& err)
{
    Dset d;
    std::vector<uint8_t> raw;
    if (!dataset(name, d, err) || !payload(d, raw, err)) return false;
    const uint64_t n = count(d.dims);
    out.resize(n);
    for (uint64_t i = 0; i < n; ++i) {
        if (d.type.cls == 1) {
            out[i] = elem_double(raw.data(), d.type, i);
        } else {
            const int64_t v = elem_int(raw.data(), d.type, i);
            out[i] = static_cast<double>(v);
            if (static_cast<int64_t>(out[i]) != v) { err = "integer not exact as a double"; return false; }
        }
    }
    if (dims) *dims = d.dims;
    return true;
}

bool Reader::attributes(const std::string& obj, std::vector<Attr>& out, std::string& err)
{
    uint64_t addr;
    if (!object(obj, addr, err)) return false;
    std::vector<Msg> msgs;
    if (!header(addr, msgs, err)) return false;
    out.clear();
    for (const Msg& m : msgs) {
        if (m.type != kMsgAttribute) continue;
        const uint8_t* p = m.data.data();
        const size_t n = m.data.size();
        if (n < 8) { err = "short attribute message"; return false; }
        const int ver = p[0];
        const uint64_t nsz = le(p + 2, 2), tsz = le(p + 4, 2), ssz = le(p + 6, 2);
        size_t pos;
        auto adv = [&](uint64_t s) { return ver == 1 ? pad8(s) : s; };
        if (ver == 1 || ver == 2) pos = 8;
        else if (ver == 3) pos = 9;
        else { err = "attribute message version " + std::to_string(ver); return false; }
        if (pos + adv(nsz) + adv(tsz) + adv(ssz) > n) { err = "short attribute message"; return false; }
        Attr a;
        a.name.assign(reinterpret_cast<const char*>(p + pos), strnlen(reinterpret_cast<const char*>(p + pos), nsz));
        pos += adv(nsz);
        if (!decode_datatype(p + pos, tsz, a.type, err)) return false;
        pos += adv(tsz);
        if (!decode_dataspace(p + pos, ssz, a.dims, err)) return false;
        pos += adv(ssz);
        uint64_t cnt;
        if (!count_ok(a.dims, cnt) || cnt * a.type.size > n) { err = "short attribute data"; return false; }
        const uint64_t bytes = cnt * a.type.size;
        if (pos + bytes > n) { err = "short attribute data"; return false; }
        a.data.assign(p + pos, p + pos + bytes);
        out.push_back(std::move(a));
    }
    return true;
}

bool Reader::has_attr(const std::string& obj, const std::string& name)
{
    std::vector<Attr> as;
    std::string err;
    if (!attributes(obj, as, err)) return false;
    for (const Attr& a : as)
        if (a.name == name) return true;
    return false;
}

bool Reader::attr_int(const std::string& obj, const std::string& name, int64_t& v, std::string& err)
{
    std::vector<Attr> as;
    if (!attributes(obj, as, err)) return false;
    for (const Attr& a : as) {
        if (a.name != name) continue;
        if (a.type.cls != 0 || count(a.dims) != 1) { err = "attribute '" + name + "' is not one integer"; return false; }
        v = elem_int(a.data.data(), a.type, 0);
        return true;
    }
    err = "no attribute '" + name + "'";
    return false;
}

bool Reader::attr_double(const std::string& obj, const std::string& name, double& v, std::string& err)
{
    std::vector<Attr> as;
    if (!attributes(obj, as, err)) return false;
    for (const Attr& a : as) {
        if (a.name != name) continue;
        if (count(a.dims) != 1) { err = "attribute '" + name + "' is not one value"; return false; }
        v = a.type.cls == 1 ? elem_double(a.data.data(), a.type, 0)
                            : static_cast<double>(elem_int(a.data.data(), a.type, 0));
        return true;
    }
    err = "no attribute '" + name + "'";
    return false;
}

// ======================= Writer =======================

void Writer::dataset(const std::string& name, const std::vector<uint64_t>& dims, Type type, const void* data)
{
    D d{name, dims, type, {}, {}};
    const uint64_t bytes = count(dims) * type.size;
    d.data.assign(static_cast<const uint8_t*>(data), static_cast<const uint8_t*>(data) + bytes);
    dsets_.push_back(std::move(d));
}

void Writer::attribute(const std::string& obj, const std::string& name, Type type, const void* value)
{
    A a{name, type, std::vector<uint8_t>(static_cast<const uint8_t*>(value), static_cast<const uint8_t*>(value) + type.size)};
    if (obj.empty()) {
        root_attrs_.push_back(std::move(a));
        return;
    }
    for (D& d : dsets_)
        if (d.name == obj) {
            d.attrs.push_back(std::move(a));
            return;
        }
    // an attribute of a dataset not added: kept on a placeholder that write() rejects
    dsets_.push_back(D{obj, {}, Type{}, {}, {std::move(a)}});
}

bool Writer::write(const std::string& path, std::string& err) const
{
    // the root group's entries, sorted by name as the symbol table requires
    std::vector<const D*> ds;
    for (const D& d : dsets_) {
        if (d.type.cls < 0) { err = "attribute on unknown dataset '" + d.name + "'"; return false; }
        if (d.name.empty() || d.name.find('/') != std::string::npos) { err = "bad dataset name '" + d.name + "'"; return false; }
        ds.push_back(&d);
    }
    std::sort(ds.begin(), ds.end(), [](const D* a, const D* b) { return std::strcmp(a->name.c_str(), b->name.c_str()) < 0; });
    for (size_t i = 1; i < ds.size(); ++i)
        if (ds[i]->name == ds[i - 1]->name) { err = "duplicate dataset '" + ds[i]->name + "'"; return false; }
    const size_t nsnod = std::max<size_t>(1, (ds.size() + 2 * kLeafK - 1) / (2 * kLeafK));
    if (nsnod > 2 * kInternalK) { err = "too many datasets for one B-tree node"; return false; }

    // local heap data: "" at 0, then the names
    Buf heap;
    heap.u(0, 8);
    std::vector<uint64_t> name_off;
    for (const D* d : ds) {
        name_off.push_back(heap.size());
        heap.raw(d->name.c_str(), d->name.size() + 1);
        heap.align8();
    }

    // addresses: superblock, root header, B-tree, heap, symbol nodes, dataset headers, data
    std::vector<HMsg> root_msgs;
    root_msgs.push_back({kMsgSymbolTable, std::vector<uint8_t>(16, 0)});
    for (const A& a : root_attrs_) root_msgs.push_back({kMsgAttribute, enc_attribute(a.name, a.type, a.value)});
    const uint64_t a_root = 96;
    const uint64_t a_btree = a_root + pad8(enc_header(root_msgs).size());
    const uint64_t a_heap = a_btree + kBtreeBytes;
    const uint64_t a_snod = a_heap + 32 + heap.size();
    uint64_t at = a_snod + nsnod * kSnodBytes;
    std::vector<std::vector<HMsg>> dmsgs(ds.size());
    std::vector<uint64_t> a_hdr(ds.size()), a_data(ds.size());
    for (size_t i = 0; i < ds.size(); ++i) {
        const D& d = *ds[i];
        auto& m = dmsgs[i];
        m.push_back({kMsgDataspace, enc_dataspace(d.dims)});
        m.push_back({kMsgDatatype, enc_datatype(d.type), 1});
        // fill value version 2: late allocation, written if set, default (zero) value
        m.push_back({kMsgFill, {2, 2, 2, 1, 0, 0, 0, 0}, 1});
        m.push_back({kMsgLayout, std::vector<uint8_t>(18, 0)});
        for (const A& a : d.attrs) m.push_back({kMsgAttribute, enc_attribute(a.name, a.type, a.value)});
        a_hdr[i] = at;
        at += pad8(enc_header(m).size());
    }
    for (size_t i = 0; i < ds.size(); ++i) {
        a_data[i] = ds[i]->data.empty() ? kUndef : at;
        at += pad8(ds[i]->data.size());
    }
    const uint64_t eof = at;
    // layout messages now that the data addresses are known
    for (size_t i = 0; i < ds.size(); ++i) {
        Buf l;
        l.u8(3);
        l.u8(1);
        l.u(a_data[i], 8);
        l.u(ds[i]->data.size(), 8);
        dmsgs[i][3].data = l.b;
    }
    {
        Buf s;
        s.u(a_btree, 8);
        s.u(a_heap, 8);
        root_msgs[0].data = s.b;
    }

    Buf out;
    // superblock version 0
    out.raw(kSig, 8);
    out.u8(0);  // superblock
    out.u8(0);  // free-space storage
    out.u8(0);  // root group symbol table entry
    out.u8(0);
    out.u8(0);  // shared header message format
    out.u8(8);  // size of offsets
    out.u8(8);  // size of lengths
    out.u8(0);
    out.u(kLeafK, 2);
    out.u(kInternalK, 2);
    out.u(0, 4);       // consistency flags
    out.u(0, 8);       // base address
    out.u(kUndef, 8);  // free-space info
    out.u(eof, 8);
    out.u(kUndef, 8);  // driver information block
    // root group symbol table entry, caching the B-tree and heap addresses
    out.u(0, 8);
    out.u(a_root, 8);
    out.u(1, 4);
    out.u(0, 4);
    out.u(a_btree, 8);
    out.u(a_heap, 8);
    // root object header
    {
        const std::vector<uint8_t> h = enc_header(root_msgs);
        out.raw(h.data(), h.size());
        out.align8();
    }
    // B-tree: one leaf over the symbol nodes; key i is the heap offset of the
    // last name of child i - 1 (key 0: the empty name)
    {
        Buf b;
        b.raw("TREE", 4);
        b.u8(0);  // group node
        b.u8(0);  // leaf level
        b.u(ds.empty() ? 0 : nsnod, 2);
        b.u(kUndef, 8);
        b.u(kUndef, 8);
        b.u(0, 8);
        if (!ds.empty())
            for (size_t s = 0; s < nsnod; ++s) {
                const size_t last = std::min(ds.size(), (s + 1) * 2 * kLeafK) - 1;
                b.u(a_snod + s * kSnodBytes, 8);
                b.u(name_off[last], 8);
            }
        b.b.resize(kBtreeBytes, 0);
        out.raw(b.b.data(), b.size());
    }
    // local heap: header, then its data (no free block: the list head is the
    // format's end-of-list value 1)
    out.raw("HEAP", 4);
    out.u8(0);
    out.u(0, 3);
    out.u(heap.size(), 8);
    out.u(1, 8);
    out.u(a_heap + 32, 8);
    out.raw(heap.b.data(), heap.size());
    // symbol nodes
    for (size_t s = 0; s < nsnod; ++s) {
        Buf n;
        n.raw("SNOD", 4);
        n.u8(1);
        n.u8(0);
        const size_t i0 = s * 2 * kLeafK, i1 = std::min(ds.size(), i0 + 2 * kLeafK);
        n.u(i1 > i0 ? i1 - i0 : 0, 2);
        for (size_t i = i0; i < i1; ++i) {
            n.u(name_off[i], 8);
            n.u(a_hdr[i], 8);
            n.u(0, 4);  // nothing cached
            n.u(0, 4);
            n.u(0, 8);
            n.u(0, 8);
        }
        n.b.resize(kSnodBytes, 0);
        out.raw(n.b.data(), n.size());
    }
    // dataset headers, then data
    for (size_t i = 0; i < ds.size(); ++i) {
        if (out.size() != a_hdr[i]) { err = "internal layout error"; return false; }
        const std::vector<uint8_t> h = enc_header(dmsgs[i]);
        out.raw(h.data(), h.size());
        out.align8();
    }
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) { err = "cannot create " + path; return false; }
    bool ok = std::fwrite(out.b.data(), 1, out.size(), f) == out.size();
    uint64_t pos = out.size();
    for (size_t i = 0; i < ds.size() && ok; ++i) {
        if (ds[i]->data.empty()) continue;
        if (pos != a_data[i]) { ok = false; break; }
        ok = std::fwrite(ds[i]->data.data(), 1, ds[i]->data.size(), f) == ds[i]->data.size();
        const uint64_t padn = pad8(ds[i]->data.size()) - ds[i]->data.size();
        static const uint8_t zeros[8] = {0};
        ok = ok && std::fwrite(zeros, 1, padn, f) == padn;
        pos += pad8(ds[i]->data.size());
    }
    ok = (std::fclose(f) == 0) && ok && pos == eof;
    if (!ok) err = "write to " + path + " failed";
    return ok;
}

}  // namespace h5
