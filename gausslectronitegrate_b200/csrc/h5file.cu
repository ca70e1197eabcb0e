// The HDF5 file format subset that the reference's files use, read and
// written without libhdf5: the sparse-ERI result file of the reference CLI
// (cli/gli_eri_integrals.c:106-163: root attributes grid_length (i64) and tol
// (f64); 1-D datasets gausslet_coeffs, integral_values (f64) and four_indices
// (i64)), which python/pymodule.c:1181-1331 loads, the coefficient file the
// CLI reads (an f64 vector attribute), and the test fixtures (test/data/*.hdf5).
//
// Host code only.  The functions behind include/hdf5_util.h keep the names,
// arguments and return values of the reference's helpers (src/hdf5_util.c);
// include/hdf5.h maps the three file calls the reference code makes (H5Fopen,
// H5Fcreate, H5Fclose) onto gli_b200_h5_fopen / _fcreate / _fclose, so that
// code written against libhdf5 for these files compiles unchanged.
//
// What is read: superblock version 0 (8-byte offsets and lengths), the root
// group's symbol table (version-1 B-tree of group nodes, symbol table nodes,
// local heap), version-1 object headers with continuation blocks, and per
// object the dataspace, datatype and layout (contiguous or compact) messages,
// plus the root group's version-1 attribute messages.  Fixed-point (1, 2, 4
// or 8 bytes, signed or not) and IEEE float (4 or 8 bytes) little-endian data
// convert to the requested memory type.
//
// What is written: the same structures, laid out the way the reference's
// libhdf5 build lays out the CLI's file (metadata in 2 KB aggregation blocks,
// raw data after them, datasets with a 256-byte object header of dataspace,
// datatype, fill value and contiguous layout messages, no modification times):
// the CLI's output for a given input is identical byte for byte wherever the
// values are.  At most 8 datasets per file (one symbol table node).
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "hdf5.h"
#include "hdf5_util.h"

namespace gli {
namespace h5 {

constexpr uint64_t UNDEF = ~(uint64_t)0;

enum Elem { E_NONE = 0, E_I64, E_I32, E_F64 };

// element type of a type id of include/hdf5.h (stored and memory types)
static Elem elem_of(hid_t t) {
    switch (t) {
        case H5T_NATIVE_DOUBLE:
        case H5T_IEEE_F64LE: return E_F64;
        case H5T_NATIVE_LLONG:
        case H5T_STD_I64LE: return E_I64;
        case H5T_NATIVE_INT:
        case H5T_STD_I32LE: return E_I32;
        default: return E_NONE;
    }
}
static size_t elem_size(Elem e) { return e == E_I32 ? 4 : 8; }

// a stored datatype: class 0 fixed point, 1 float; size in bytes
struct DType {
    int cls = -1;
    int size = 0;
    bool is_signed = true;
};

struct Item {
    std::string name;
    DType type;
    std::vector<uint64_t> dims;  // empty: scalar
    std::vector<uint8_t> raw;    // little-endian stored elements
    uint64_t count() const {
        uint64_t n = 1;
        for (uint64_t d : dims) n *= d;
        return n;
    }
};

struct File {
    std::string path;
    bool writing = false;
    std::vector<Item> attrs, dsets;
};

static std::mutex g_mu;
static std::map<hid_t, std::unique_ptr<File>> g_files;
static hid_t g_next = 1;

static File* find(hid_t id) {
    auto it = g_files.find(id);
    return it == g_files.end() ? nullptr : it->second.get();
}

// ---------------------------------------------------------------------------
// conversion between stored elements and memory elements
static double load_as_double(const DType& t, const uint8_t* p) {
    if (t.cls == 1) {
        if (t.size == 8) {
            double v;
            memcpy(&v, p, 8);
            return v;
        }
        float f;
        memcpy(&f, p, 4);
        return f;
    }
    uint64_t u = 0;
    memcpy(&u, p, t.size);
    if (t.is_signed && t.size < 8 && (u >> (8 * t.size - 1)) & 1) u |= ~(uint64_t)0 << (8 * t.size);
    return t.is_signed ? (double)(int64_t)u : (double)u;
}
static int64_t load_as_int(const DType& t, const uint8_t* p) {
    if (t.cls == 1) return (int64_t)load_as_double(t, p);
    uint64_t u = 0;
    memcpy(&u, p, t.size);
    if (t.is_signed && t.size < 8 && (u >> (8 * t.size - 1)) & 1) u |= ~(uint64_t)0 << (8 * t.size);
    return (int64_t)u;
}
static bool convert_out(const Item& it, Elem mem, void* out) {
    if (mem == E_NONE || it.type.cls < 0) return false;
    const uint64_t n = it.count();
    if (it.raw.size() < n * (uint64_t)it.type.size) return false;
    for (uint64_t k = 0; k < n; ++k) {
        const uint8_t* p = it.raw.data() + k * it.type.size;
        if (mem == E_F64)
            ((double*)out)[k] = load_as_double(it.type, p);
        else if (mem == E_I64)
            ((int64_t*)out)[k] = load_as_int(it.type, p);
        else
            ((int32_t*)out)[k] = (int32_t)load_as_int(it.type, p);
    }
    return true;
}
static bool convert_in(Item& it, Elem store, Elem input, const void* in) {
    if (store == E_NONE || input == E_NONE) return false;
    it.type.cls = store == E_F64 ? 1 : 0;
    it.type.size = (int)elem_size(store);
    it.type.is_signed = true;
    const uint64_t n = it.count();
    it.raw.assign(n * it.type.size, 0);
    for (uint64_t k = 0; k < n; ++k) {
        uint8_t* p = it.raw.data() + k * it.type.size;
        double dv = 0;
        int64_t iv = 0;
        if (input == E_F64) {
            dv = ((const double*)in)[k];
            iv = (int64_t)dv;
        } else {
            iv = input == E_I64 ? ((const int64_t*)in)[k] : ((const int32_t*)in)[k];
            dv = (double)iv;
        }
        if (store == E_F64)
            memcpy(p, &dv, 8);
        else if (store == E_I64)
            memcpy(p, &iv, 8);
        else {
            const int32_t v = (int32_t)iv;
            memcpy(p, &v, 4);
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// reading
struct Reader {
    std::vector<uint8_t> d;
    bool ok = true;
    uint64_t u(uint64_t off, int n) {
        if (off + n > d.size()) {
            ok = false;
            return 0;
        }
        uint64_t v = 0;
        memcpy(&v, d.data() + off, n);
        return v;
    }
    bool sig(uint64_t off, const char* s) { return off + 4 <= d.size() && memcmp(d.data() + off, s, 4) == 0; }
    std::string cstr(uint64_t off) {
        std::string s;
        while (off < d.size() && d[off]) s.push_back((char)d[off++]);
        if (off >= d.size()) ok = false;
        return s;
    }
};

static DType parse_dtype(Reader& r, uint64_t p) {
    DType t;
    const int cv = (int)r.u(p, 1);
    t.cls = cv & 0x0f;
    const int bits0 = (int)r.u(p + 1, 1);
    t.size = (int)r.u(p + 4, 4);
    if (t.cls == 0) {
        t.is_signed = (bits0 & 0x08) != 0;
        if (bits0 & 1) t.cls = -1;  // big-endian: not read
        if (t.size != 1 && t.size != 2 && t.size != 4 && t.size != 8) t.cls = -1;
    } else if (t.cls == 1) {
        if ((bits0 & 1) || (t.size != 4 && t.size != 8)) t.cls = -1;
    } else {
        t.cls = -1;
    }
    return t;
}

// dataspace message body at p: version 1 or 2, rank, dims
static std::vector<uint64_t> parse_dspace(Reader& r, uint64_t p) {
    const int ver = (int)r.u(p, 1), rank = (int)r.u(p + 1, 1);
    std::vector<uint64_t> dims;
    const uint64_t d0 = ver == 1 ? p + 8 : p + 4;
    for (int k = 0; k < rank; ++k) dims.push_back(r.u(d0 + 8 * k, 8));
    return dims;
}

// messages of a version-1 object header, following continuation blocks
struct Msg {
    int type;
    uint64_t body, size;
};
static std::vector<Msg> object_messages(Reader& r, uint64_t addr) {
    std::vector<Msg> out;
    if (r.u(addr, 1) != 1) {
        r.ok = false;
        return out;
    }
    const uint64_t nmsg = r.u(addr + 2, 2), hsize = r.u(addr + 8, 4);
    std::vector<std::pair<uint64_t, uint64_t>> chunks{{addr + 16, hsize}};
    for (size_t c = 0; c < chunks.size() && r.ok && out.size() < nmsg; ++c) {
        uint64_t p = chunks[c].first;
        const uint64_t end = p + chunks[c].second;
        while (p + 8 <= end && r.ok && out.size() < nmsg) {
            const int type = (int)r.u(p, 2);
            const uint64_t size = r.u(p + 2, 2);
            if (type == 0x10) chunks.push_back({r.u(p + 8, 8), r.u(p + 16, 8)});
            out.push_back({type, p + 8, size});
            p += 8 + size;
        }
        if (chunks.size() > 64) r.ok = false;
    }
    return out;
}

static bool read_dataset(Reader& r, const std::string& name, uint64_t ohdr, Item& it) {
    it.name = name;
    uint64_t addr = UNDEF, size = 0;
    bool have_layout = false;
    for (const Msg& m : object_messages(r, ohdr)) {
        if (m.type == 0x1) it.dims = parse_dspace(r, m.body);
        if (m.type == 0x3) it.type = parse_dtype(r, m.body);
        if (m.type == 0x8) {
            const int ver = (int)r.u(m.body, 1), cls = (int)r.u(m.body + 1, 1);
            if (ver != 3) continue;
            if (cls == 1) {  // contiguous
                addr = r.u(m.body + 2, 8);
                size = r.u(m.body + 10, 8);
                have_layout = true;
            } else if (cls == 0) {  // compact: the data follow the size
                size = r.u(m.body + 2, 2);
                addr = m.body + 4;
                have_layout = true;
            }
        }
    }
    if (!have_layout || it.type.cls < 0 || !r.ok) return false;
    const uint64_t need = it.count() * (uint64_t)it.type.size;
    if (addr == UNDEF) {  // never written: the fill value, zeros
        it.raw.assign(need, 0);
        return true;
    }
    if (size < need || addr + need > r.d.size()) return false;
    it.raw.assign(r.d.begin() + addr, r.d.begin() + addr + need);
    return true;
}

// a version-1 attribute message body
static bool read_attribute(Reader& r, uint64_t p, Item& it) {
    if (r.u(p, 1) != 1) return false;
    const uint64_t nlen = r.u(p + 2, 2), tlen = r.u(p + 4, 2), slen = r.u(p + 6, 2);
    auto pad8 = [](uint64_t x) { return (x + 7) / 8 * 8; };
    uint64_t q = p + 8;
    it.name = r.cstr(q);
    q += pad8(nlen);
    it.type = parse_dtype(r, q);
    q += pad8(tlen);
    it.dims = parse_dspace(r, q);
    q += pad8(slen);
    const uint64_t need = it.count() * (uint64_t)it.type.size;
    if (it.type.cls < 0 || q + need > r.d.size() || !r.ok) return false;
    it.raw.assign(r.d.begin() + q, r.d.begin() + q + need);
    return true;
}

// symbol table entries below a version-1 B-tree node of group type
static void walk_group_btree(Reader& r, uint64_t node, uint64_t heap_data, std::vector<std::pair<std::string, uint64_t>>& out,
                             int depth) {
    if (!r.sig(node, "TREE") || r.u(node + 4, 1) != 0 || depth > 16) {
        r.ok = false;
        return;
    }
    const int level = (int)r.u(node + 5, 1);
    const uint64_t n = r.u(node + 6, 2);
    for (uint64_t k = 0; k < n && r.ok; ++k) {
        const uint64_t child = r.u(node + 24 + 8 + 16 * k, 8);
        if (level > 0) {
            walk_group_btree(r, child, heap_data, out, depth + 1);
            continue;
        }
        if (!r.sig(child, "SNOD")) {
            r.ok = false;
            return;
        }
        const uint64_t ns = r.u(child + 6, 2);
        for (uint64_t e = 0; e < ns; ++e) {
            const uint64_t ent = child + 8 + 40 * e;
            out.push_back({r.cstr(heap_data + r.u(ent, 8)), r.u(ent + 8, 8)});
        }
    }
}

static bool parse_file(const std::string& path, File& f) {
    Reader r;
    FILE* fp = fopen(path.c_str(), "rb");
    if (!fp) return false;
    fseek(fp, 0, SEEK_END);
    const long len = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    r.d.resize(len > 0 ? (size_t)len : 0);
    const size_t got = r.d.empty() ? 0 : fread(r.d.data(), 1, r.d.size(), fp);
    fclose(fp);
    static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    if (got != r.d.size() || r.d.size() < 96 || memcmp(r.d.data(), sig, 8) != 0) return false;
    if (r.u(8, 1) != 0 || r.u(13, 1) != 8 || r.u(14, 1) != 8) return false;  // superblock 0, 8-byte sizes
    const uint64_t root = r.u(56 + 8, 8);
    uint64_t btree = UNDEF, heap = UNDEF;
    for (const Msg& m : object_messages(r, root)) {
        if (m.type == 0x11) {
            btree = r.u(m.body, 8);
            heap = r.u(m.body + 8, 8);
        }
        if (m.type == 0xc) {
            Item it;
            if (read_attribute(r, m.body, it)) f.attrs.push_back(std::move(it));
        }
    }
    if (btree == UNDEF || !r.sig(heap, "HEAP") || !r.ok) return false;
    const uint64_t heap_data = r.u(heap + 24, 8);
    std::vector<std::pair<std::string, uint64_t>> entries;
    walk_group_btree(r, btree, heap_data, entries, 0);
    for (const auto& e : entries) {
        Item it;
        if (read_dataset(r, e.first, e.second, it)) f.dsets.push_back(std::move(it));
    }
    return r.ok;
}

// ---------------------------------------------------------------------------
// writing
struct Writer {
    std::vector<uint8_t> d;
    void put(uint64_t off, uint64_t v, int n) {
        if (off + n > d.size()) d.resize(off + n, 0);
        memcpy(d.data() + off, &v, n);
    }
    void put_bytes(uint64_t off, const void* p, size_t n) {
        if (off + n > d.size()) d.resize(off + n, 0);
        if (n) memcpy(d.data() + off, p, n);
    }
};

static uint64_t pad8(uint64_t x) { return (x + 7) / 8 * 8; }

// datatype message body; returns its unpadded size
static std::vector<uint8_t> dtype_bytes(const DType& t) {
    std::vector<uint8_t> b;
    auto u8 = [&](uint64_t v, int n) {
        for (int k = 0; k < n; ++k) b.push_back((uint8_t)(v >> (8 * k)));
    };
    if (t.cls == 1) {  // IEEE float, little-endian, implied leading mantissa bit
        const bool dbl = t.size == 8;
        u8(0x11, 1);
        u8(0x20, 1);
        u8(dbl ? 63 : 31, 1);
        u8(0, 1);
        u8(t.size, 4);
        u8(0, 2);                  // bit offset
        u8(8 * t.size, 2);         // precision
        u8(dbl ? 52 : 23, 1);      // exponent location
        u8(dbl ? 11 : 8, 1);       // exponent size
        u8(0, 1);                  // mantissa location
        u8(dbl ? 52 : 23, 1);      // mantissa size
        u8(dbl ? 1023 : 127, 4);   // exponent bias
    } else {  // fixed point, little-endian, two's complement
        u8(0x10, 1);
        u8(t.is_signed ? 0x08 : 0x00, 1);
        u8(0, 1);
        u8(0, 1);
        u8(t.size, 4);
        u8(0, 2);
        u8(8 * t.size, 2);
    }
    return b;
}

// dataspace message body (version 1): scalar, or the dims with equal maxima
static std::vector<uint8_t> dspace_bytes(const std::vector<uint64_t>& dims) {
    std::vector<uint8_t> b(8, 0);
    b[0] = 1;
    b[1] = (uint8_t)dims.size();
    b[2] = dims.empty() ? 0 : 1;
    for (int pass = 0; pass < (dims.empty() ? 0 : 2); ++pass)
        for (uint64_t v : dims)
            for (int k = 0; k < 8; ++k) b.push_back((uint8_t)(v >> (8 * k)));
    return b;
}

static std::vector<uint8_t> attribute_body(const Item& a) {
    const std::vector<uint8_t> t = dtype_bytes(a.type), sp = dspace_bytes(a.dims);
    const uint64_t nlen = a.name.size() + 1;
    std::vector<uint8_t> b(8 + pad8(nlen) + pad8(t.size()) + pad8(sp.size()), 0);
    b[0] = 1;
    b[2] = (uint8_t)nlen;
    b[3] = (uint8_t)(nlen >> 8);
    b[4] = (uint8_t)t.size();
    b[6] = (uint8_t)sp.size();
    memcpy(b.data() + 8, a.name.c_str(), a.name.size());
    memcpy(b.data() + 8 + pad8(nlen), t.data(), t.size());
    memcpy(b.data() + 8 + pad8(nlen) + pad8(t.size()), sp.data(), sp.size());
    b.insert(b.end(), a.raw.begin(), a.raw.end());
    b.resize(pad8(b.size()), 0);
    return b;
}

static void put_msg(Writer& w, uint64_t& p, int type, const std::vector<uint8_t>& body, int flags) {
    w.put(p, type, 2);
    w.put(p + 2, body.size(), 2);
    w.put(p + 4, flags, 1);
    w.put_bytes(p + 8, body.data(), body.size());
    p += 8 + body.size();
}

// file space: metadata in 2 KB aggregation blocks, raw data at the end of file
struct Space {
    uint64_t eof = 0, blk_end = 0, cursor = 0;
    uint64_t meta(uint64_t n) {
        if (cursor + n <= blk_end) {
            const uint64_t a = cursor;
            cursor += n;
            return a;
        }
        const uint64_t a = eof;
        blk_end = eof + std::max<uint64_t>(2048, n);
        cursor = a + n;
        eof = blk_end;
        return a;
    }
    uint64_t raw(uint64_t n) {
        const uint64_t a = eof;
        eof += n;
        return a;
    }
};

static bool serialize(const File& f, std::vector<uint8_t>& out, std::string& why) {
    constexpr uint64_t ROOT = 96, BTREE = 136, HEAP = 680, HEAP_DATA = 712;
    constexpr int LEAF_K = 4, NODE_K = 16;
    if (f.dsets.size() > 2 * LEAF_K) {
        why = "at most 8 datasets per file";
        return false;
    }
    // local heap: the empty name, then each name padded to 8 bytes; a free block after
    std::vector<uint64_t> name_off;
    uint64_t used = 8;
    for (const Item& it : f.dsets) {
        name_off.push_back(used);
        used += pad8(it.name.size() + 1);
    }
    const uint64_t heap_size = std::max<uint64_t>(88, used + 16);
    const uint64_t cont = HEAP_DATA + heap_size;
    std::vector<std::vector<uint8_t>> attr_bodies;
    uint64_t cont_len = 8 + 16;  // the symbol table message
    for (const Item& a : f.attrs) {
        attr_bodies.push_back(attribute_body(a));
        cont_len += 8 + attr_bodies.back().size();
    }
    Space sp;
    sp.blk_end = 2048;
    sp.cursor = cont + cont_len;
    if (sp.cursor > sp.blk_end) sp.blk_end = sp.cursor;
    sp.eof = sp.blk_end;
    // creation order: per dataset its object header, the symbol table node at the
    // first link, the raw data
    std::vector<uint64_t> ohdr(f.dsets.size()), data(f.dsets.size());
    uint64_t snod = UNDEF;
    for (size_t k = 0; k < f.dsets.size(); ++k) {
        ohdr[k] = sp.meta(16 + 256);
        if (k == 0) snod = sp.meta(8 + 2 * LEAF_K * 40);
        const uint64_t nbytes = f.dsets[k].raw.size();
        data[k] = nbytes ? sp.raw(nbytes) : UNDEF;
    }
    // an unused tail of the last metadata block at the end of the file is dropped
    const uint64_t eof = (sp.eof == sp.blk_end) ? sp.cursor : sp.eof;

    Writer w;
    w.d.assign(eof, 0);
    static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    w.put_bytes(0, sig, 8);
    // versions 0 (superblock, free space, root symbol table, shared headers), sizes 8 / 8
    w.put(13, 8, 1);
    w.put(14, 8, 1);
    w.put(16, LEAF_K, 2);
    w.put(18, NODE_K, 2);
    w.put(24, 0, 8);       // base address
    w.put(32, UNDEF, 8);   // free-space info
    w.put(40, eof, 8);     // end of file
    w.put(48, UNDEF, 8);   // driver info
    w.put(56, 0, 8);       // root entry: link name offset
    w.put(64, ROOT, 8);    //             object header
    w.put(72, 1, 4);       //             cache type: symbol table scratch
    w.put(80, BTREE, 8);
    w.put(88, HEAP, 8);
    // root object header: one continuation message in its first chunk
    w.put(ROOT, 1, 1);
    w.put(ROOT + 2, 2 + f.attrs.size(), 2);
    w.put(ROOT + 4, 1, 4);
    w.put(ROOT + 8, 24, 4);
    {
        uint64_t p = ROOT + 16;
        std::vector<uint8_t> b(16);
        memcpy(b.data(), &cont, 8);
        memcpy(b.data() + 8, &cont_len, 8);
        put_msg(w, p, 0x10, b, 0);
        p = cont;
        std::vector<uint8_t> st(16);
        const uint64_t bt = BTREE, hp = HEAP;
        memcpy(st.data(), &bt, 8);
        memcpy(st.data() + 8, &hp, 8);
        put_msg(w, p, 0x11, st, 0);
        for (const auto& ab : attr_bodies) put_msg(w, p, 0xc, ab, 0);
    }
    // B-tree (group nodes, level 0): keys are heap offsets of names
    std::vector<size_t> order(f.dsets.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = k;
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return f.dsets[a].name < f.dsets[b].name; });
    w.put_bytes(BTREE, "TREE", 4);
    w.put(BTREE + 6, f.dsets.empty() ? 0 : 1, 2);
    w.put(BTREE + 8, UNDEF, 8);
    w.put(BTREE + 16, UNDEF, 8);
    if (!f.dsets.empty()) {
        w.put(BTREE + 24, 0, 8);
        w.put(BTREE + 32, snod, 8);
        w.put(BTREE + 40, name_off[order.back()], 8);
    }
    // local heap
    w.put_bytes(HEAP, "HEAP", 4);
    w.put(HEAP + 8, heap_size, 8);
    w.put(HEAP + 16, used, 8);  // free block right after the names
    w.put(HEAP + 24, HEAP_DATA, 8);
    for (size_t k = 0; k < f.dsets.size(); ++k)
        w.put_bytes(HEAP_DATA + name_off[k], f.dsets[k].name.c_str(), f.dsets[k].name.size());
    w.put(HEAP_DATA + used, 1, 8);  // no next free block
    w.put(HEAP_DATA + used + 8, heap_size - used, 8);
    // symbol table node, entries sorted by name
    if (!f.dsets.empty()) {
        w.put_bytes(snod, "SNOD", 4);
        w.put(snod + 4, 1, 1);
        w.put(snod + 6, f.dsets.size(), 2);
        for (size_t e = 0; e < order.size(); ++e) {
            w.put(snod + 8 + 40 * e, name_off[order[e]], 8);
            w.put(snod + 16 + 40 * e, ohdr[order[e]], 8);
        }
    }
    // datasets
    for (size_t k = 0; k < f.dsets.size(); ++k) {
        const Item& it = f.dsets[k];
        const uint64_t h = ohdr[k];
        w.put(h, 1, 1);
        w.put(h + 2, 5, 2);
        w.put(h + 4, 1, 4);
        w.put(h + 8, 256, 4);
        uint64_t p = h + 16;
        put_msg(w, p, 0x1, dspace_bytes(it.dims), 0);
        std::vector<uint8_t> t = dtype_bytes(it.type);
        t.resize(pad8(t.size()), 0);
        put_msg(w, p, 0x3, t, 1);
        put_msg(w, p, 0x5, std::vector<uint8_t>{2, 2, 2, 1, 0, 0, 0, 0}, 1);  // fill value: late allocation, default
        std::vector<uint8_t> lay(24, 0);
        lay[0] = 3;
        lay[1] = 1;  // contiguous
        const uint64_t nbytes = it.raw.size();
        memcpy(lay.data() + 2, &data[k], 8);
        memcpy(lay.data() + 10, &nbytes, 8);
        put_msg(w, p, 0x8, lay, 0);
        const uint64_t left = h + 16 + 256 - p;
        if (left < 8) {
            why = "dataset header overflow";
            return false;
        }
        put_msg(w, p, 0x0, std::vector<uint8_t>(left - 8, 0), 0);
        if (nbytes) w.put_bytes(data[k], it.raw.data(), nbytes);
    }
    out.swap(w.d);
    return true;
}

}  // namespace h5
}  // namespace gli

using gli::h5::File;
using gli::h5::Item;

extern "C" {

hid_t gli_b200_h5_fopen(const char* name, unsigned flags, hid_t fapl) {
    (void)flags;
    (void)fapl;
    if (!name) return -1;
    auto f = std::make_unique<File>();
    f->path = name;
    if (!gli::h5::parse_file(f->path, *f)) return -1;
    std::lock_guard<std::mutex> lk(gli::h5::g_mu);
    const hid_t id = gli::h5::g_next++;
    gli::h5::g_files[id] = std::move(f);
    return id;
}

hid_t gli_b200_h5_fcreate(const char* name, unsigned flags, hid_t fcpl, hid_t fapl) {
    (void)flags;
    (void)fcpl;
    (void)fapl;
    if (!name) return -1;
    FILE* fp = fopen(name, "wb");  // H5F_ACC_TRUNC: the file exists, empty, from here on
    if (!fp) return -1;
    fclose(fp);
    auto f = std::make_unique<File>();
    f->path = name;
    f->writing = true;
    std::lock_guard<std::mutex> lk(gli::h5::g_mu);
    const hid_t id = gli::h5::g_next++;
    gli::h5::g_files[id] = std::move(f);
    return id;
}

herr_t gli_b200_h5_fclose(hid_t file) {
    std::unique_ptr<File> f;
    {
        std::lock_guard<std::mutex> lk(gli::h5::g_mu);
        auto it = gli::h5::g_files.find(file);
        if (it == gli::h5::g_files.end()) return -1;
        f = std::move(it->second);
        gli::h5::g_files.erase(it);
    }
    if (!f->writing) return 0;
    std::vector<uint8_t> bytes;
    std::string why;
    if (!gli::h5::serialize(*f, bytes, why)) {
        fprintf(stderr, "writing '%s' failed: %s\n", f->path.c_str(), why.c_str());
        return -1;
    }
    FILE* fp = fopen(f->path.c_str(), "wb");
    if (!fp) return -1;
    const size_t n = fwrite(bytes.data(), 1, bytes.size(), fp);
    return (fclose(fp) == 0 && n == bytes.size()) ? 0 : -1;
}

}  // extern "C"

namespace {
const Item* lookup(hid_t file, const char* name, bool attr) {
    File* f = gli::h5::find(file);
    if (!f || !name) return nullptr;
    for (const Item& it : attr ? f->attrs : f->dsets)
        if (it.name == name) return &it;
    return nullptr;
}
}  // namespace

herr_t get_hdf5_dataset_ndims(hid_t file, const char* name, int* ndims) {
    std::lock_guard<std::mutex> lk(gli::h5::g_mu);
    const Item* it = lookup(file, name, false);
    if (!it) {
        fprintf(stderr, "'H5Dopen' for '%s' failed\n", name ? name : "(null)");
        return -1;
    }
    *ndims = (int)it->dims.size();
    return 0;
}

herr_t get_hdf5_dataset_dims(hid_t file, const char* name, hsize_t* dims) {
    std::lock_guard<std::mutex> lk(gli::h5::g_mu);
    const Item* it = lookup(file, name, false);
    if (!it) {
        fprintf(stderr, "'H5Dopen' for '%s' failed\n", name ? name : "(null)");
        return -1;
    }
    for (size_t k = 0; k < it->dims.size(); ++k) dims[k] = (hsize_t)it->dims[k];
    return 0;
}

herr_t read_hdf5_dataset(hid_t file, const char* name, hid_t mem_type, void* data) {
    std::lock_guard<std::mutex> lk(gli::h5::g_mu);
    const Item* it = lookup(file, name, false);
    if (!it) {
        fprintf(stderr, "'H5Dopen' for '%s' failed\n", name ? name : "(null)");
        return -1;
    }
    if (!gli::h5::convert_out(*it, gli::h5::elem_of(mem_type), data)) {
        fprintf(stderr, "'H5Dread' for '%s' failed, return value: %d\n", name, -1);
        return -1;
    }
    return 0;
}

herr_t write_hdf5_dataset(hid_t file, const char* name, int degree, const hsize_t dims[], hid_t mem_type_store,
                          hid_t mem_type_input, const void* data) {
    std::lock_guard<std::mutex> lk(gli::h5::g_mu);
    File* f = gli::h5::find(file);
    if (!f || !f->writing || !name || degree < 0 || degree > 32) {
        fprintf(stderr, "'H5Dcreate' for '%s' failed\n", name ? name : "(null)");
        return -1;
    }
    Item it;
    it.name = name;
    for (int k = 0; k < degree; ++k) it.dims.push_back(dims[k]);
    if (!gli::h5::convert_in(it, gli::h5::elem_of(mem_type_store), gli::h5::elem_of(mem_type_input), data)) {
        fprintf(stderr, "'H5Dwrite' for '%s' failed, return value: %d\n", name, -1);
        return -1;
    }
    for (const Item& o : f->dsets)
        if (o.name == it.name) {
            fprintf(stderr, "'H5Dcreate' for '%s' failed\n", name);
            return -1;
        }
    f->dsets.push_back(std::move(it));
    return 0;
}

herr_t get_hdf5_attribute_dims(hid_t file, const char* name, hsize_t* dims) {
    std::lock_guard<std::mutex> lk(gli::h5::g_mu);
    const Item* it = lookup(file, name, true);
    if (!it) {
        fprintf(stderr, "'H5Aopen' for '%s' failed\n", name ? name : "(null)");
        return -1;
    }
    for (size_t k = 0; k < it->dims.size(); ++k) dims[k] = (hsize_t)it->dims[k];
    return 0;
}

herr_t read_hdf5_attribute(hid_t file, const char* name, hid_t mem_type, void* data) {
    std::lock_guard<std::mutex> lk(gli::h5::g_mu);
    const Item* it = lookup(file, name, true);
    if (!it) {
        fprintf(stderr, "'H5Aopen' for '%s' failed\n", name ? name : "(null)");
        return -1;
    }
    if (!gli::h5::convert_out(*it, gli::h5::elem_of(mem_type), data)) {
        fprintf(stderr, "'H5Aread' for '%s' failed, return value: %d\n", name, -1);
        return -1;
    }
    return 0;
}

static herr_t write_attribute(hid_t file, const char* name, const std::vector<uint64_t>& dims, hid_t store,
                              hid_t input, const void* data) {
    std::lock_guard<std::mutex> lk(gli::h5::g_mu);
    File* f = gli::h5::find(file);
    if (!f || !f->writing || !name) {
        fprintf(stderr, "'H5Acreate' for '%s' failed\n", name ? name : "(null)");
        return -1;
    }
    Item it;
    it.name = name;
    it.dims = dims;
    if (!gli::h5::convert_in(it, gli::h5::elem_of(store), gli::h5::elem_of(input), data)) {
        fprintf(stderr, "'H5Awrite' for '%s' failed\n", name);
        return -1;
    }
    for (Item& o : f->attrs)
        if (o.name == it.name) {
            o = std::move(it);
            return 0;
        }
    f->attrs.push_back(std::move(it));
    return 0;
}

herr_t write_hdf5_scalar_attribute(hid_t file, const char* name, hid_t mem_type_store, hid_t mem_type_input,
                                   const void* data) {
    return write_attribute(file, name, {}, mem_type_store, mem_type_input, data);
}

herr_t write_hdf5_vector_attribute(hid_t file, const char* name, hid_t mem_type_store, hid_t mem_type_input,
                                   const glong length, const void* data) {
    if (length < 0) return -1;
    return write_attribute(file, name, {(uint64_t)length}, mem_type_store, mem_type_input, data);
}

// ---------------------------------------------------------------------------
// Monotonic ticks for the reference's drivers (include/timing.h): nanoseconds
// of CLOCK_MONOTONIC, as the reference's src/timing.c counts them on Linux.
#include <time.h>

#include "timing.h"

int64_t get_time_ticks(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return 1000000000LL * (int64_t)t.tv_sec + (int64_t)t.tv_nsec;
}

int64_t get_tick_resolution(void) { return 1000000000LL; }
