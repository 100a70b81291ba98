// cl_h5.hpp — a minimal HDF5 file writer for the output files, written from
// the HDF5 File Format Specification (version 3.0); header-only C++17.
//
// It writes the same subset, byte for byte, as crysplight_b200/hdf5.py: one
// root group holding contiguous datasets and scalar root attributes, the
// structures the reference writes with HDF5.jl (src/output.jl:10-32):
//   * superblock version 2 (8-byte offsets and lengths, Jenkins lookup3
//     checksum);
//   * root group: version-2 object header with compact link storage (Link
//     Info, Group Info, one hard-link Link message per dataset) and one
//     Attribute message (version 3) per attribute;
//   * datasets: version-2 object headers with Dataspace (version 2), Datatype
//     (version 1), Fill Value (version 3) and Data Layout (version 3,
//     contiguous) messages; raw data after the headers, 8-byte aligned.
// Arrays are given in Julia's column-major order with their Julia dimensions;
// the dataspace lists them reversed, as HDF5.jl does, so an (nx, ny, n) array
// reads as (n, ny, nx) in h5py.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace clh5 {

// Bob Jenkins' lookup3 hashlittle (public domain, 2006): the checksum of the
// version-2 structures.
inline uint32_t lookup3(const uint8_t* k, size_t length, uint32_t initval = 0)
{
    auto rot = [](uint32_t x, int r) { return (x << r) | (x >> (32 - r)); };
    auto word = [](const uint8_t* p) {
        return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
    };
    uint32_t a, b, c;
    a = b = c = 0xdeadbeefu + (uint32_t)length + initval;
    while (length > 12) {
        a += word(k); b += word(k + 4); c += word(k + 8);
        a -= c; a ^= rot(c, 4);  c += b;
        b -= a; b ^= rot(a, 6);  a += c;
        c -= b; c ^= rot(b, 8);  b += a;
        a -= c; a ^= rot(c, 16); c += b;
        b -= a; b ^= rot(a, 19); a += c;
        c -= b; c ^= rot(b, 4);  b += a;
        length -= 12;
        k += 12;
    }
    if (length == 0) return c;
    uint8_t tail[12] = {0};
    std::memcpy(tail, k, length);
    a += word(tail); b += word(tail + 4); c += word(tail + 8);
    c ^= b; c -= rot(b, 14);
    a ^= c; a -= rot(c, 11);
    b ^= a; b -= rot(a, 25);
    c ^= b; c -= rot(b, 16);
    a ^= c; a -= rot(c, 4);
    b ^= a; b -= rot(a, 14);
    c ^= b; c -= rot(b, 24);
    return c;
}

using Bytes = std::vector<uint8_t>;

inline void put(Bytes& o, uint64_t v, int n)
{
    for (int i = 0; i < n; ++i) o.push_back((uint8_t)(v >> (8 * i)));
}
inline void put(Bytes& o, const Bytes& b) { o.insert(o.end(), b.begin(), b.end()); }

// Element types of datasets and attributes.
enum class Type { I8, U8, I16, U16, I32, U32, I64, U64, F32, F64, Str };

inline int type_size(Type t)
{
    switch (t) {
    case Type::I8: case Type::U8: return 1;
    case Type::I16: case Type::U16: return 2;
    case Type::I32: case Type::U32: case Type::F32: return 4;
    case Type::I64: case Type::U64: case Type::F64: return 8;
    default: return 0;
    }
}

// Datatype message body (version 1); strlen > 0 for a fixed-length
// null-terminated UTF-8 string.
inline Bytes datatype(Type t, uint32_t strlen = 0)
{
    Bytes o;
    if (t == Type::Str) {
        o.push_back((1 << 4) | 3);
        o.push_back(0x10); o.push_back(0); o.push_back(0);
        put(o, strlen, 4);
        return o;
    }
    const int size = type_size(t);
    if (t == Type::F32 || t == Type::F64) {
        const bool d = t == Type::F64;
        o.push_back((1 << 4) | 1);
        o.push_back(0x20); o.push_back(d ? 63 : 31); o.push_back(0);
        put(o, (uint64_t)size, 4);
        put(o, 0, 2);                       // bit offset
        put(o, (uint64_t)(8 * size), 2);    // precision
        o.push_back(d ? 52 : 23);           // exponent location
        o.push_back(d ? 11 : 8);            // exponent size
        o.push_back(0);                     // mantissa location
        o.push_back(d ? 52 : 23);           // mantissa size
        put(o, d ? 1023 : 127, 4);          // exponent bias
        return o;
    }
    const bool is_signed = t == Type::I8 || t == Type::I16 || t == Type::I32 || t == Type::I64;
    o.push_back((1 << 4) | 0);
    o.push_back(is_signed ? 0x08 : 0); o.push_back(0); o.push_back(0);
    put(o, (uint64_t)size, 4);
    put(o, 0, 2);
    put(o, (uint64_t)(8 * size), 2);
    return o;
}

// Dataspace message body (version 2); no dims = scalar.
inline Bytes dataspace(const std::vector<uint64_t>& dims)
{
    Bytes o;
    o.push_back(2);
    o.push_back((uint8_t)dims.size());
    o.push_back(0);
    o.push_back(dims.empty() ? 0 : 1);
    for (uint64_t d : dims) put(o, d, 8);
    return o;
}

inline Bytes message(int type, const Bytes& body, int flags = 0)
{
    Bytes o;
    o.push_back((uint8_t)type);
    put(o, body.size(), 2);
    o.push_back((uint8_t)flags);
    put(o, body);
    return o;
}

// Version-2 object header with one chunk (chunk size in 4 bytes); with
// attr_phase, attribute phase-change values (max compact 64, min dense 6).
inline Bytes object_header(const Bytes& msgs, bool attr_phase)
{
    Bytes o = {'O', 'H', 'D', 'R', 2, (uint8_t)(0x02 | (attr_phase ? 0x10 : 0))};
    if (attr_phase) { put(o, 64, 2); put(o, 6, 2); }
    put(o, msgs.size(), 4);
    put(o, msgs);
    put(o, lookup3(o.data(), o.size()), 4);
    return o;
}

constexpr int MSG_DATASPACE = 0x01, MSG_LINK_INFO = 0x02, MSG_DATATYPE = 0x03, MSG_FILL = 0x05;
constexpr int MSG_LINK = 0x06, MSG_LAYOUT = 0x08, MSG_GROUP_INFO = 0x0A, MSG_ATTRIBUTE = 0x0C;
constexpr uint64_t UNDEF = 0xFFFFFFFFFFFFFFFFull;

struct Dataset {
    std::string name;
    Type type;
    std::vector<uint64_t> julia_dims;   // Julia dimensions (column-major data)
    Bytes raw;                          // little-endian elements, column-major
};

struct Attribute {
    std::string name;
    Type type;
    Bytes raw;                          // one little-endian scalar, or the string's bytes
};

inline Attribute attr_str(const std::string& name, const std::string& v)
{
    return {name, Type::Str, Bytes(v.begin(), v.end())};
}
template <typename T>
inline Attribute attr_num(const std::string& name, Type t, T v)
{
    Bytes b(sizeof(T));
    std::memcpy(b.data(), &v, sizeof(T));
    return {name, t, b};
}

class Writer {
public:
    void add_dataset(Dataset d) { ds_.push_back(std::move(d)); }
    void add_attribute(Attribute a) { at_.push_back(std::move(a)); }

    // Write the file; throws std::runtime_error on I/O errors.
    void write(const std::string& path) const
    {
        const uint64_t sb_size = 48;
        std::vector<uint64_t> zeros(ds_.size(), 0);
        const uint64_t root_size = root_header(zeros).size();
        uint64_t pos = sb_size + root_size;
        std::vector<uint64_t> hdr_addr, data_addr;
        for (const Dataset& d : ds_) {
            hdr_addr.push_back(pos);
            pos += ds_header(d, 0).size();
        }
        for (const Dataset& d : ds_) {
            pos = (pos + 7) & ~(uint64_t)7;
            data_addr.push_back(pos);
            pos += d.raw.size();
        }
        const uint64_t eof = pos;
        Bytes root = root_header(hdr_addr);
        if (root.size() != root_size) throw std::runtime_error("hdf5: root header size changed");
        Bytes out = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n', 2, 8, 8, 0};
        put(out, 0, 8);
        put(out, UNDEF, 8);
        put(out, eof, 8);
        put(out, sb_size, 8);
        put(out, lookup3(out.data(), out.size()), 4);
        put(out, root);
        for (size_t i = 0; i < ds_.size(); ++i)
            put(out, ds_header(ds_[i], ds_[i].raw.empty() ? UNDEF : data_addr[i]));
        for (size_t i = 0; i < ds_.size(); ++i) {
            out.resize(data_addr[i], 0);
            put(out, ds_[i].raw);
        }
        if (out.size() != eof) throw std::runtime_error("hdf5: size mismatch");
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) throw std::runtime_error("cannot open " + path + " for writing");
        const size_t n = std::fwrite(out.data(), 1, out.size(), f);
        const int rc = std::fclose(f);
        if (n != out.size() || rc != 0) throw std::runtime_error("write failed: " + path);
    }

private:
    std::vector<Dataset> ds_;
    std::vector<Attribute> at_;

    static Bytes ds_header(const Dataset& d, uint64_t addr)
    {
        std::vector<uint64_t> dims(d.julia_dims.rbegin(), d.julia_dims.rend());
        Bytes fill = {3, 0x0A};
        Bytes layout = {3, 1};
        put(layout, addr, 8);
        put(layout, d.raw.size(), 8);
        Bytes m = message(MSG_DATASPACE, dataspace(dims));
        put(m, message(MSG_DATATYPE, datatype(d.type), 0x01));
        put(m, message(MSG_FILL, fill));
        put(m, message(MSG_LAYOUT, layout));
        return object_header(m, false);
    }

    static Bytes attribute(const Attribute& a)
    {
        Bytes nm(a.name.begin(), a.name.end());
        nm.push_back(0);
        Bytes data = a.raw, dt;
        if (a.type == Type::Str) {
            data.push_back(0);
            dt = datatype(Type::Str, (uint32_t)data.size());
        } else {
            dt = datatype(a.type);
        }
        Bytes sp = dataspace({});
        Bytes o = {3, 0};
        put(o, nm.size(), 2);
        put(o, dt.size(), 2);
        put(o, sp.size(), 2);
        o.push_back(1);                     // UTF-8 name
        put(o, nm);
        put(o, dt);
        put(o, sp);
        put(o, data);
        return o;
    }

    Bytes root_header(const std::vector<uint64_t>& addrs) const
    {
        Bytes li = {0, 0};
        put(li, UNDEF, 8);
        put(li, UNDEF, 8);
        Bytes gi = {0, 0x01};
        put(gi, 64, 2);
        put(gi, 6, 2);
        Bytes m = message(MSG_LINK_INFO, li);
        put(m, message(MSG_GROUP_INFO, gi));
        for (size_t i = 0; i < ds_.size(); ++i) {
            const std::string& n = ds_[i].name;
            if (n.size() > 255) throw std::runtime_error("hdf5: dataset names are limited to 255 bytes");
            Bytes l = {1, 0x10, 1, (uint8_t)n.size()};
            l.insert(l.end(), n.begin(), n.end());
            put(l, addrs[i], 8);
            put(m, message(MSG_LINK, l));
        }
        for (const Attribute& a : at_) put(m, message(MSG_ATTRIBUTE, attribute(a)));
        return object_header(m, true);
    }
};

}  // namespace clh5
