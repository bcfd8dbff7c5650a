// host_h5.cpp -- minimal reader for the reference's gw_input.h5 (no libhdf5 needed).
//
// Reads exactly what the reference's reader consumes (src/hdf5_input.cpp:192-212): the float64
// datasets /mo_energy (nmo), /eri_mo (nmo^4, C order) and /vxc_mo (nmo^2), and the root
// attributes nocc (integer) and fermi_energy (float64), with the reference's validation
// (src/hdf5_input.cpp:174-188).  Supported subset of the HDF5 file format (as written by h5py
// with the default "earliest" format): superblock v0/v1, version-1 object headers with
// continuation blocks, symbol-table groups (v1 B-tree + SNOD + local heap), dataspace v1/v2,
// IEEE little-endian float and integer datatypes, compact or contiguous layout (v1-v4) and
// attribute messages v1-v3.  Anything else fails with GWB200_IO_ERROR naming the feature.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "internal.cuh"

namespace gwb200 {
namespace {

[[noreturn]] void io_fail(const std::string& m) { fail(GWB200_IO_ERROR, "gw_input.h5: " + m); }

struct Message {
    uint16_t type;
    uint8_t flags;
    std::vector<uint8_t> data;
};

struct TypeInfo {
    int cls = -1;      // 0 fixed point, 1 float
    size_t size = 0;
    bool little = true;
    bool is_signed = true;
};

struct Dataset {
    std::vector<uint64_t> dims;
    TypeInfo type;
    int layout = -1;  // 0 compact, 1 contiguous
    uint64_t address = UINT64_MAX;
    uint64_t nbytes = 0;
    std::vector<uint8_t> compact;
};

class Reader {
public:
    explicit Reader(const std::string& path) : fp_(std::fopen(path.c_str(), "rb"), &std::fclose) {
        if (!fp_) fail(GWB200_IO_ERROR, "Could not open HDF5 input file: " + path);
        std::fseek(fp_.get(), 0, SEEK_END);
        size_ = static_cast<uint64_t>(std::ftell(fp_.get()));
        parse_superblock();
    }

    uint64_t root_header() const { return root_header_; }

    std::vector<Message> object_messages(uint64_t addr) {
        std::vector<Message> msgs;
        std::vector<uint8_t> pre = read(addr, 16);
        if (pre[0] != 1) {
            if (std::memcmp(pre.data(), "OHDR", 4) == 0) io_fail("version-2 object headers are not supported");
            io_fail("unknown object header version " + std::to_string(pre[0]));
        }
        const uint16_t nmsgs = u16(pre.data() + 2);
        const uint32_t hsize = u32(pre.data() + 8);
        std::vector<std::pair<uint64_t, uint64_t>> blocks{{addr + 16, hsize}};
        size_t bi = 0;
        while (bi < blocks.size() && msgs.size() < nmsgs) {
            const auto [baddr, blen] = blocks[bi++];
            std::vector<uint8_t> b = read(baddr, blen);
            size_t off = 0;
            while (off + 8 <= b.size() && msgs.size() < nmsgs) {
                Message m;
                m.type = u16(&b[off]);
                const uint16_t sz = u16(&b[off + 2]);
                m.flags = b[off + 4];
                if (off + 8 + sz > b.size()) io_fail("truncated object header message");
                m.data.assign(b.begin() + static_cast<long>(off + 8), b.begin() + static_cast<long>(off + 8 + sz));
                off += 8 + sz;
                if (m.type == 0x10) {
                    blocks.emplace_back(uoff(m.data.data()), ulen(m.data.data() + so_));
                }
                msgs.push_back(std::move(m));
            }
        }
        return msgs;
    }

    std::map<std::string, uint64_t> group_members(const std::vector<Message>& msgs) {
        for (const auto& m : msgs) {
            if (m.type == 0x11) {
                const uint64_t btree = uoff(m.data.data());
                const uint64_t heap = uoff(m.data.data() + so_);
                std::vector<uint8_t> h = read(heap, 8 + 2 * sl_ + so_);
                if (std::memcmp(h.data(), "HEAP", 4) != 0) io_fail("bad local heap signature");
                const uint64_t heap_size = ulen(h.data() + 8);
                const uint64_t heap_data = uoff(h.data() + 8 + 2 * sl_);
                heap_ = read(heap_data, heap_size);
                std::map<std::string, uint64_t> out;
                walk_btree(btree, out, 0);
                return out;
            }
        }
        io_fail("root group has no symbol table (new-style link storage is not supported)");
    }

    Dataset dataset(uint64_t header) {
        Dataset d;
        for (const auto& m : object_messages(header)) {
            if (m.flags & 0x02) {
                if (m.type == 0x01 || m.type == 0x03 || m.type == 0x08) io_fail("shared dataset messages are not supported");
                continue;
            }
            if (m.type == 0x01) d.dims = dataspace(m.data.data(), m.data.size());
            else if (m.type == 0x03) d.type = datatype(m.data.data(), m.data.size());
            else if (m.type == 0x08) layout(m.data, d);
        }
        if (d.type.cls < 0) io_fail("dataset without datatype");
        if (d.type.cls != 0 && d.type.cls != 1) io_fail("unsupported dataset datatype class " + std::to_string(d.type.cls));
        if (d.layout < 0) io_fail("dataset without a compact or contiguous layout");
        return d;
    }

    // Reads the dataset as float64 into out (count elements).
    void read_f64(const Dataset& d, double* out, uint64_t count, const std::string& name) {
        if (d.type.cls != 1 || d.type.size != 8 || !d.type.little) io_fail(name + " is not little-endian float64");
        const uint64_t bytes = count * 8;
        if (d.layout == 0) {
            if (d.compact.size() < bytes) io_fail(name + ": compact data too short");
            std::memcpy(out, d.compact.data(), bytes);
            return;
        }
        if (d.address == UINT64_MAX) {
            std::memset(out, 0, bytes);  // never written: HDF5 default fill value 0
            return;
        }
        read_into(d.address, reinterpret_cast<uint8_t*>(out), bytes);
    }

    // Reads elements [first, first + count) of the dataset (C order) as float64: one contiguous
    // run of the file (contiguous layout) or of the compact data.
    void read_f64_range(const Dataset& d, uint64_t first, uint64_t count, double* out, const std::string& name) {
        if (d.type.cls != 1 || d.type.size != 8 || !d.type.little) io_fail(name + " is not little-endian float64");
        uint64_t total = 1;
        for (auto x : d.dims) total *= x;
        if (first > total || count > total - first) io_fail(name + ": element range beyond the dataset");
        const uint64_t bytes = count * 8;
        if (d.layout == 0) {
            if (d.compact.size() < (first + count) * 8) io_fail(name + ": compact data too short");
            std::memcpy(out, d.compact.data() + first * 8, bytes);
            return;
        }
        if (d.address == UINT64_MAX) {
            std::memset(out, 0, bytes);
            return;
        }
        read_into(d.address + first * 8, reinterpret_cast<uint8_t*>(out), bytes);
    }

    // Root attributes: name -> (type, raw bytes).
    std::map<std::string, std::pair<TypeInfo, std::vector<uint8_t>>> attributes(const std::vector<Message>& msgs) {
        std::map<std::string, std::pair<TypeInfo, std::vector<uint8_t>>> out;
        for (const auto& m : msgs) {
            if (m.type != 0x0C) continue;
            const uint8_t* p = m.data.data();
            const uint8_t ver = p[0];
            const uint16_t nsz = u16(p + 2), tsz = u16(p + 4), ssz = u16(p + 6);
            size_t off = 8;
            if (ver == 3) off = 9;
            else if (ver != 1 && ver != 2) io_fail("unsupported attribute message version");
            auto pad = [&](size_t x) { return ver == 1 ? (x + 7) / 8 * 8 : x; };
            const std::string name(reinterpret_cast<const char*>(p + off), strnlen(reinterpret_cast<const char*>(p + off), nsz));
            off += pad(nsz);
            const TypeInfo t = datatype(p + off, tsz);
            off += pad(tsz);
            if (t.cls != 0 && t.cls != 1) continue;  // strings, compounds ...: not consumed
            const std::vector<uint64_t> dims = dataspace(p + off, ssz);
            off += pad(ssz);
            uint64_t count = 1;
            for (auto x : dims) count *= x;
            const size_t bytes = static_cast<size_t>(count * t.size);
            if (off + bytes > m.data.size()) io_fail("truncated attribute " + name);
            out[name] = {t, std::vector<uint8_t>(p + off, p + off + bytes)};
        }
        return out;
    }

private:
    std::unique_ptr<FILE, int (*)(FILE*)> fp_;
    uint64_t size_ = 0;
    uint64_t base_ = 0;
    int so_ = 8, sl_ = 8;
    uint64_t root_header_ = 0;
    std::vector<uint8_t> heap_;

    static uint16_t u16(const uint8_t* p) { return static_cast<uint16_t>(p[0] | (p[1] << 8)); }
    static uint32_t u32(const uint8_t* p) { return p[0] | (p[1] << 8) | (p[2] << 16) | (static_cast<uint32_t>(p[3]) << 24); }
    static uint64_t un(const uint8_t* p, int n) {
        uint64_t v = 0;
        for (int i = n - 1; i >= 0; --i) v = (v << 8) | p[i];
        return v;
    }
    uint64_t uoff(const uint8_t* p) const { return un(p, so_); }
    uint64_t ulen(const uint8_t* p) const { return un(p, sl_); }

    void read_into(uint64_t addr, uint8_t* dst, uint64_t n) {
        const uint64_t a = addr + base_;
        if (a > size_ || n > size_ - a) io_fail("address beyond end of file");
        if (std::fseek(fp_.get(), static_cast<long>(a), SEEK_SET) != 0) io_fail("seek failed");
        if (std::fread(dst, 1, n, fp_.get()) != n) io_fail("short read");
    }
    std::vector<uint8_t> read(uint64_t addr, uint64_t n) {
        std::vector<uint8_t> b(n);
        read_into(addr, b.data(), n);
        return b;
    }

    void parse_superblock() {
        static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
        uint64_t at = 0;
        for (;; at = at ? at * 2 : 512) {
            if (at + 8 > size_) io_fail("HDF5 signature not found");
            uint8_t s[8];
            if (std::fseek(fp_.get(), static_cast<long>(at), SEEK_SET) != 0 || std::fread(s, 1, 8, fp_.get()) != 8)
                io_fail("cannot read superblock");
            if (std::memcmp(s, sig, 8) == 0) break;
        }
        std::vector<uint8_t> sb(128);
        if (std::fseek(fp_.get(), static_cast<long>(at), SEEK_SET) != 0) io_fail("seek failed");
        const size_t got = std::fread(sb.data(), 1, sb.size(), fp_.get());
        if (got < 56) io_fail("truncated superblock");
        const int ver = sb[8];
        if (ver > 1) io_fail("superblock version " + std::to_string(ver) + " is not supported");
        so_ = sb[13];
        sl_ = sb[14];
        if (so_ != 8 || sl_ != 8) io_fail("only 8-byte offsets and lengths are supported");
        size_t off = ver == 0 ? 24 : 28;
        base_ = uoff(&sb[off]);
        off += 4 * so_;
        root_header_ = uoff(&sb[off + so_]);  // root symbol table entry: name offset, header address
    }

    void walk_btree(uint64_t addr, std::map<std::string, uint64_t>& out, int depth) {
        if (depth > 32) io_fail("group B-tree too deep");
        std::vector<uint8_t> h = read(addr, 8 + 2 * so_);
        if (std::memcmp(h.data(), "TREE", 4) != 0) io_fail("bad B-tree signature");
        const int level = h[5];
        const int used = u16(&h[6]);
        std::vector<uint8_t> body = read(addr + 8 + 2 * so_, static_cast<uint64_t>(used) * (sl_ + so_) + sl_);
        for (int i = 0; i < used; ++i) {
            const uint64_t child = uoff(&body[static_cast<size_t>(i) * (sl_ + so_) + sl_]);
            if (level > 0) {
                walk_btree(child, out, depth + 1);
                continue;
            }
            std::vector<uint8_t> sn = read(child, 8);
            if (std::memcmp(sn.data(), "SNOD", 4) != 0) io_fail("bad symbol table node");
            const int nsym = u16(&sn[6]);
            const uint64_t esz = 2 * so_ + 24;
            std::vector<uint8_t> ents = read(child + 8, esz * nsym);
            for (int e = 0; e < nsym; ++e) {
                const uint8_t* ep = &ents[e * esz];
                const uint64_t name_off = uoff(ep);
                if (name_off >= heap_.size()) io_fail("link name outside the local heap");
                const char* nm = reinterpret_cast<const char*>(&heap_[name_off]);
                out[std::string(nm, strnlen(nm, heap_.size() - name_off))] = uoff(ep + so_);
            }
        }
    }

    std::vector<uint64_t> dataspace(const uint8_t* p, size_t n) const {
        if (n < 8) io_fail("truncated dataspace");
        const int ver = p[0], nd = p[1];
        size_t off = (ver == 1) ? 8 : (ver == 2 ? 4 : 0);
        if (off == 0) io_fail("unsupported dataspace version");
        if (off + static_cast<size_t>(nd) * sl_ > n) io_fail("truncated dataspace dims");
        std::vector<uint64_t> dims(static_cast<size_t>(nd));
        for (int i = 0; i < nd; ++i) dims[static_cast<size_t>(i)] = ulen(p + off + static_cast<size_t>(i) * sl_);
        return dims;
    }

    static TypeInfo datatype(const uint8_t* p, size_t n) {
        if (n < 8) io_fail("truncated datatype");
        TypeInfo t;
        t.cls = p[0] & 0x0F;
        t.little = (p[1] & 0x01) == 0;
        t.is_signed = (p[1] & 0x08) != 0;
        t.size = u32(p + 4);
        return t;  // callers check the class they need (integer 0, float 1)
    }

    void layout(const std::vector<uint8_t>& m, Dataset& d) const {
        const uint8_t* p = m.data();
        const int ver = p[0];
        if (ver >= 3) {
            const int cls = p[1];
            if (cls == 0) {
                const uint16_t sz = u16(p + 2);
                d.layout = 0;
                d.compact.assign(p + 4, p + 4 + sz);
            } else if (cls == 1) {
                d.layout = 1;
                d.address = uoff(p + 2);
                d.nbytes = ulen(p + 2 + so_);
            } else {
                io_fail("chunked or virtual dataset layouts are not supported");
            }
        } else if (ver == 1 || ver == 2) {
            const int cls = p[2];
            if (cls == 1) {
                d.layout = 1;
                d.address = uoff(p + 8);
            } else if (cls == 0) {
                const int nd = p[1];
                const size_t off = 8 + 4 * static_cast<size_t>(nd);
                const uint32_t sz = u32(p + off);
                d.layout = 0;
                d.compact.assign(p + off + 4, p + off + 4 + sz);
            } else {
                io_fail("chunked dataset layouts are not supported");
            }
        } else {
            io_fail("unsupported layout message version");
        }
    }
};

// The three datasets and two attributes of a validated gw_input.h5.
struct Input {
    Dataset dmo, deri, dvxc;
    uint64_t nmo = 0;
    int64_t nocc = 0;
    double fermi = 0.0;
};

Input open_input(Reader& r) {
    const auto root_msgs = r.object_messages(r.root_header());
    const auto members = r.group_members(root_msgs);
    auto need = [&](const char* name) {
        auto it = members.find(name);
        if (it == members.end()) io_fail(std::string("Could not open HDF5 dataset: /") + name);
        return r.dataset(it->second);
    };
    const Dataset dmo = need("mo_energy");
    const Dataset deri = need("eri_mo");
    const Dataset dvxc = need("vxc_mo");
    if (dmo.dims.size() != 1) io_fail("HDF5 dataset /mo_energy has rank " + std::to_string(dmo.dims.size()) + ", expected 1");
    if (deri.dims.size() != 4) io_fail("HDF5 dataset /eri_mo is not a rank-4 tensor");
    if (dvxc.dims.size() != 2) io_fail("HDF5 dataset /vxc_mo is not a matrix");
    const uint64_t nmo = dmo.dims[0];
    if (nmo == 0) io_fail("HDF5 input error: mo_energy is empty");
    for (auto x : deri.dims)
        if (x != nmo) io_fail("HDF5 input error: eri_mo shape does not match mo_energy length");
    if (dvxc.dims[0] != nmo || dvxc.dims[1] != nmo) io_fail("HDF5 input error: vxc_mo shape does not match mo_energy length");

    const auto attrs = r.attributes(root_msgs);
    auto ia = attrs.find("nocc");
    auto fa = attrs.find("fermi_energy");
    if (ia == attrs.end()) io_fail("Could not open HDF5 file attribute: nocc");
    if (fa == attrs.end()) io_fail("Could not open HDF5 file attribute: fermi_energy");
    int64_t nocc = 0;
    {
        const auto& [t, b] = ia->second;
        if (t.cls != 0 || !t.little || t.size == 0 || t.size > 8 || b.size() < t.size) io_fail("nocc is not a little-endian integer");
        uint64_t v = 0;
        for (size_t i = t.size; i-- > 0;) v = (v << 8) | b[i];
        if (t.is_signed && t.size < 8 && (v >> (8 * t.size - 1)) & 1) v |= ~uint64_t{0} << (8 * t.size);
        nocc = static_cast<int64_t>(v);
    }
    double fermi = 0.0;
    {
        const auto& [t, b] = fa->second;
        if (t.cls != 1 || !t.little || b.size() < t.size) io_fail("fermi_energy is not a little-endian float");
        if (t.size == 8) {
            std::memcpy(&fermi, b.data(), 8);
        } else if (t.size == 4) {
            float f;
            std::memcpy(&f, b.data(), 4);
            fermi = f;
        } else {
            io_fail("fermi_energy has an unsupported float size");
        }
    }
    if (nocc < 0) io_fail("HDF5 input error: nocc attribute is negative");
    if (nocc == 0 || static_cast<uint64_t>(nocc) >= nmo) io_fail("HDF5 input error: nocc must be in [1, nmo-1]");
    return Input{dmo, deri, dvxc, nmo, nocc, fermi};
}

} // namespace

void read_gw_input_h5(const std::string& path, int64_t* nmo_out, int64_t* nocc_out, double* fermi_out, double* mo,
                      double* eri, double* vxc) {
    Reader r(path);
    const Input in = open_input(r);
    const uint64_t nmo = in.nmo;
    *nmo_out = static_cast<int64_t>(nmo);
    *nocc_out = in.nocc;
    *fermi_out = in.fermi;
    if (mo) r.read_f64(in.dmo, mo, nmo, "/mo_energy");
    if (eri) r.read_f64(in.deri, eri, nmo * nmo * nmo * nmo, "/eri_mo");
    if (vxc) r.read_f64(in.dvxc, vxc, nmo * nmo, "/vxc_mo");
}

// The slices of the file's ERI tensor that the screening path reads for a known state list, read
// straight from /eri_mo without the nmo^4 tensor in memory (the layouts gwb200_load_system_slices
// takes):
//   vph[(j nvir + b) n + i nvir + a]        = eri[j, nocc + b, i, nocc + a]   (n x n)
//   panel[(t nmo + k) n + i nvir + a]       = eri[states[t], k, i, nocc + a]  ((nstates nmo) x n)
//   xdiag[p nocc + i]                       = eri[p, i, p, i]                 (nmo x nocc)
//   vxc_diag[p]                             = vxc_mo[p, p]
// Each (j, b) row of V and each (t, k) row of the panel is one read of the contiguous run
// eri[., ., 0:nocc, 0:nmo] (nocc nmo doubles), scattered to the nvir-long runs the layout keeps.
void read_gw_input_h5_slices(const std::string& path, const int64_t* states, int64_t nstates, int64_t* nmo_out,
                             int64_t* nocc_out, double* fermi_out, double* mo, double* vph, double* panel,
                             double* xdiag, double* vxc_diag) {
    Reader r(path);
    const Input in = open_input(r);
    const uint64_t nmo = in.nmo, nocc = static_cast<uint64_t>(in.nocc), nvir = nmo - nocc, n = nocc * nvir;
    *nmo_out = static_cast<int64_t>(nmo);
    *nocc_out = in.nocc;
    *fermi_out = in.fermi;
    if (!mo && !vph && !panel && !xdiag && !vxc_diag) return;  // size query
    if (!mo || !vph || !panel || !xdiag || !vxc_diag) fail(GWB200_BAD_ARGUMENT, "null output array");
    if (!states || nstates <= 0) fail(GWB200_BAD_SHAPE, "at least one state is required");
    for (int64_t t = 0; t < nstates; ++t)
        if (states[t] < 0 || static_cast<uint64_t>(states[t]) >= nmo) fail(GWB200_BAD_SHAPE, "Selected state is out of range");
    r.read_f64(in.dmo, mo, nmo, "/mo_energy");
    std::vector<double> run(static_cast<size_t>(nocc * nmo));
    auto cut = [&](uint64_t p, uint64_t q, double* row) {  // row[i nvir + a] = eri[p, q, i, nocc + a]
        r.read_f64_range(in.deri, (p * nmo + q) * nmo * nmo, nocc * nmo, run.data(), "/eri_mo");
        for (uint64_t i = 0; i < nocc; ++i) std::memcpy(row + i * nvir, run.data() + i * nmo + nocc, nvir * sizeof(double));
    };
    for (uint64_t j = 0; j < nocc; ++j)
        for (uint64_t b = 0; b < nvir; ++b) cut(j, nocc + b, vph + (j * nvir + b) * n);
    for (int64_t t = 0; t < nstates; ++t)
        for (uint64_t k = 0; k < nmo; ++k)
            cut(static_cast<uint64_t>(states[t]), k, panel + (static_cast<uint64_t>(t) * nmo + k) * n);
    for (uint64_t p = 0; p < nmo; ++p)
        for (uint64_t i = 0; i < nocc; ++i)
            r.read_f64_range(in.deri, ((p * nmo + i) * nmo + p) * nmo + i, 1, xdiag + p * nocc + i, "/eri_mo");
    for (uint64_t p = 0; p < nmo; ++p) r.read_f64_range(in.dvxc, p * nmo + p, 1, vxc_diag + p, "/vxc_mo");
}

} // namespace gwb200
