// Snapshot writer with the layout of alsfvm::io::NetCDFWriter
// (alsfvm/src/io/NetCDFWriter.cpp:32-146), host code.
//
// The reference writes NetCDF-4 through libnetcdf, which this library does
// not link; this writer produces the classic NetCDF format (version 2,
// 64-bit offsets), which the same readers open (libnetcdf, ncdump, xarray,
// scipy.io.netcdf_file), with the reference's content:
//   dimensions  t = 1, x = nx, y = ny, z = nz   (NetCDFWriter.cpp:50-53, 85-97)
//   variables   time (double, t)                 the snapshot's time
//               one double variable per conserved variable, named as the
//               reference names them (rho, mx, [my, [mz,]] E;
//               alsfvm/src/equation/euler/Euler.cpp:20-75), dimensions
//               (x, y, z), holding the interior cells in the order
//               Volume::copyInternalCells produces (x fastest,
//               HostMemory.cpp:239-258) — the same bytes under the same
//               dimension names as the reference's files
//   attributes  global text attributes given by the caller
// File names: <base>_<snapshot>.nc (alsfvm/src/io/io_utils.cpp:34-40).
// Numbers in the file are big-endian, as the format prescribes.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "als_b200.h"

namespace als {
int report_error(int code, const char* msg);
}

namespace {

class Header {
public:
    void u32(uint32_t v) {
        for (int s = 24; s >= 0; s -= 8) {
            bytes.push_back(uint8_t(v >> s));
        }
    }
    void u64(uint64_t v) {
        for (int s = 56; s >= 0; s -= 8) {
            bytes.push_back(uint8_t(v >> s));
        }
    }
    void name(const std::string& s) {
        u32(uint32_t(s.size()));
        text(s);
    }
    void text(const std::string& s) {
        bytes.insert(bytes.end(), s.begin(), s.end());
        while (bytes.size() % 4) {
            bytes.push_back(0);
        }
    }
    std::vector<uint8_t> bytes;
};

constexpr uint32_t kDimension = 0x0A;
constexpr uint32_t kVariable = 0x0B;
constexpr uint32_t kAttribute = 0x0C;
constexpr uint32_t kChar = 2;
constexpr uint32_t kDouble = 6;

void put_be_doubles(std::FILE* f, const double* v, size_t count) {
    std::vector<uint8_t> buf(8 * 4096);
    for (size_t i = 0; i < count; i += 4096) {
        const size_t k = count - i < 4096 ? count - i : 4096;
        for (size_t j = 0; j < k; ++j) {
            uint64_t u;
            std::memcpy(&u, v + i + j, 8);
            for (int b = 0; b < 8; ++b) {
                buf[8 * j + b] = uint8_t(u >> (56 - 8 * b));
            }
        }
        std::fwrite(buf.data(), 1, 8 * k, f);
    }
}

} // namespace

extern "C" int als_write_netcdf(const char* path, int dimension, const int* n, int nvar,
    const char* const* names, const double* const* interior, double time, int nattr,
    const char* const* attr_names, const char* const* attr_values) {
    if (!path || dimension < 1 || dimension > 3 || !n || nvar < 1 || !names || !interior ||
        nattr < 0 || (nattr > 0 && (!attr_names || !attr_values))) {
        return als::report_error(ALS_E_INVALID, "invalid NetCDF writer arguments");
    }
    uint32_t dims[3];
    for (int d = 0; d < 3; ++d) {
        dims[d] = uint32_t(d < dimension ? n[d] : 1);
        if (d < dimension && n[d] < 1) {
            return als::report_error(ALS_E_INVALID, "invalid grid size");
        }
    }
    const uint64_t cells = uint64_t(dims[0]) * dims[1] * dims[2];
    const uint64_t vsize = cells * 8;

    // header with begin offsets filled in once its size is known (the
    // offsets are fixed-size fields, so a first pass gives the length)
    auto build = [&](uint64_t data_begin) {
        Header h;
        h.bytes = {'C', 'D', 'F', 2};   // classic format, version 2 (64-bit offsets)
        h.u32(0);                        // numrecs
        h.u32(kDimension);
        h.u32(4);
        h.name("t");
        h.u32(1);
        const char* dn[3] = {"x", "y", "z"};
        for (int d = 0; d < 3; ++d) {
            h.name(dn[d]);
            h.u32(dims[d]);
        }
        if (nattr > 0) {
            h.u32(kAttribute);
            h.u32(uint32_t(nattr));
            for (int a = 0; a < nattr; ++a) {
                const std::string value = attr_values[a] ? attr_values[a] : "";
                h.name(attr_names[a] ? attr_names[a] : "");
                h.u32(kChar);
                h.u32(uint32_t(value.size()));
                h.text(value);
            }
        } else {
            h.u32(0);
            h.u32(0);
        }
        h.u32(kVariable);
        h.u32(uint32_t(1 + nvar));
        uint64_t begin = data_begin;
        // time(t)
        h.name("time");
        h.u32(1);
        h.u32(0);
        h.u32(0);
        h.u32(0);             // no variable attributes
        h.u32(kDouble);
        h.u32(8);
        h.u64(begin);
        begin += 8;
        for (int v = 0; v < nvar; ++v) {
            h.name(names[v] ? names[v] : "");
            h.u32(3);
            h.u32(1);
            h.u32(2);
            h.u32(3);
            h.u32(0);
            h.u32(0);
            h.u32(kDouble);
            h.u32(vsize < 0xFFFFFFFFull ? uint32_t(vsize) : 0xFFFFFFFFu);
            h.u64(begin);
            begin += vsize;
        }
        return h;
    };
    const size_t header_size = build(0).bytes.size();
    const Header h = build(header_size);

    std::FILE* f = std::fopen(path, "wb");
    if (!f) {
        return als::report_error(ALS_E_INVALID, (std::string("cannot open ") + path).c_str());
    }
    std::fwrite(h.bytes.data(), 1, h.bytes.size(), f);
    put_be_doubles(f, &time, 1);
    for (int v = 0; v < nvar; ++v) {
        put_be_doubles(f, interior[v], cells);
    }
    const bool ok = std::ferror(f) == 0;
    if (std::fclose(f) != 0 || !ok) {
        return als::report_error(ALS_E_INVALID, (std::string("write failed: ") + path).c_str());
    }
    return ALS_OK;
}
