// Writes a small file through crysplight_b200/csrc/cl_h5.hpp, for the test
// that compares it byte for byte with crysplight_b200/hdf5.py's writer.
//   h5_writer_check <path>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "../../crysplight_b200/csrc/cl_h5.hpp"

int main(int argc, char** argv)
{
    if (argc != 2) return 2;
    using namespace clh5;
    Writer w;
    // counts: Julia (3, 2, 4) UInt32, column-major values 7*k + 1
    Dataset c{"counts", Type::U32, {3, 2, 4}, Bytes(3 * 2 * 4 * 4)};
    for (uint32_t k = 0; k < 24; ++k) {
        const uint32_t v = 7 * k + 1;
        std::memcpy(c.raw.data() + 4 * k, &v, 4);
    }
    // first_time_ns: Julia (3, 2) Float32, k * 0.5 with Inf at k = 4
    Dataset f{"first_time_ns", Type::F32, {3, 2}, Bytes(6 * 4)};
    for (int k = 0; k < 6; ++k) {
        const float v = k == 4 ? INFINITY : 0.5f * (float)k;
        std::memcpy(f.raw.data() + 4 * k, &v, 4);
    }
    Dataset e{"empty", Type::F64, {0}, Bytes()};
    // small integer types of events.h5: int8 (2, 3), int16 (3,), uint16 (3,)
    Dataset i8{"int_type", Type::I8, {2, 3}, Bytes{0xFF, 0, 1, 2, 0x80, 0x7F}};
    Dataset i16{"n_int", Type::I16, {3}, Bytes{0xFF, 0xFF, 0x02, 0x00, 0x00, 0x80}};
    Dataset u16{"maps", Type::U16, {3}, Bytes{0x01, 0x00, 0xFF, 0xFF, 0x34, 0x12}};
    w.add_dataset(c);
    w.add_dataset(f);
    w.add_dataset(e);
    w.add_dataset(i8);
    w.add_dataset(i16);
    w.add_dataset(u16);
    w.add_attribute(attr_str("tag", "h5 check"));
    w.add_attribute(attr_num("n_photons", Type::I64, (int64_t)1000000));
    w.add_attribute(attr_num("bin_ns", Type::F32, 100.0f));
    w.add_attribute(attr_num("nbins", Type::I32, (int32_t)80));
    w.add_attribute(attr_num("flag", Type::U8, (uint8_t)1));
    w.add_attribute(attr_num("big", Type::U64, (uint64_t)0xFFFFFFFFFFFFFFF0ull));
    w.add_attribute(attr_num("u32", Type::U32, (uint32_t)4000000000u));
    w.add_attribute(attr_num("sigma_alpha_deg", Type::F64, 1.3));
    w.add_attribute(attr_str("empty_str", ""));
    try {
        w.write(argv[1]);
    } catch (const std::exception& ex) {
        std::fprintf(stderr, "%s\n", ex.what());
        return 1;
    }
    return 0;
}
