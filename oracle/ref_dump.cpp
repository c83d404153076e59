// Oracle-side dump driver around the unmodified ASZ reference compressor.
//
// Test infrastructure only: it is built by oracle/Makefile from the reference sources where
// they lie and is never linked into the product. It compiles c_codes/s1_compress.cpp as is,
// with `main` renamed, and runs that main. The one hook is an explicit specialisation of the
// reference's `write_compressed_stream<float>` (c_codes/s1_compress.cpp:142-151): it writes
// the .asz exactly as the reference does and, next to it, `<asz>.dump` holding the internal
// arrays the compressor left in its `param_c` (c_codes/asz_core/asz_param.hpp:131-245):
//   "ASZDUMP1"
//   u64 layer_num+1, then per QB stream: u64 count, count x int32      (qb_vec_vec)
//   u64 t_count, t_count x int64                                       (t_int_vec)
//   u64 n, n x float32                                                 (compressed_data)
//   f32 min_val, f32 max_val, f32 abs_eb, f32 default_slope, u8 force_quintic
//   u64 plan length, plan bytes (comma-separated predictor_vec)
// The .asz it writes must equal the plain reference binary's; the tests check that.
#include "asz_core/asz_param.hpp"

template<typename T> void write_compressed_stream(const asz::param_c<T> &param);
template<> void write_compressed_stream<float>(const asz::param_c<float> &param);

#define main asz_reference_s1_compress_main
#include "s1_compress.cpp"
#undef main

template<typename V>
static void put(std::ofstream &o, const V &v) { o.write(reinterpret_cast<const char *>(&v), sizeof(V)); }

template<> void write_compressed_stream<float>(const asz::param_c<float> &param)
{
    {
        std::ofstream output(param.compressed_data_path, std::ios::binary);
        if (!output)
            throw std::runtime_error("cannot open compressed output: " + param.compressed_data_path);
        output.write(reinterpret_cast<const char *>(param.zstd_bs_vec.data()), param.zstd_bs_vec.size());
        if (!output)
            throw std::runtime_error("cannot write compressed output: " + param.compressed_data_path);
    }
    std::ofstream d(param.compressed_data_path + ".dump", std::ios::binary);
    d.write("ASZDUMP1", 8);
    put(d, (uint64_t)param.qb_vec_vec.size());
    for (auto &v : param.qb_vec_vec) {
        put(d, (uint64_t)v.size());
        d.write(reinterpret_cast<const char *>(v.data()), v.size() * sizeof(int32_t));
    }
    put(d, (uint64_t)param.t_int_vec.size());
    d.write(reinterpret_cast<const char *>(param.t_int_vec.data()), param.t_int_vec.size() * sizeof(int64_t));
    put(d, (uint64_t)param.compressed_data.size());
    d.write(reinterpret_cast<const char *>(param.compressed_data.data()), param.compressed_data.size() * sizeof(float));
    put(d, param.min_val);
    put(d, param.max_val);
    put(d, param.abs_eb);
    put(d, param.default_slope);
    put(d, (uint8_t)param.force_quintic);
    std::string plan;
    for (size_t i = 0; i < param.predictor_vec.size(); i++)
        plan += (i ? "," : "") + param.predictor_vec[i];
    put(d, (uint64_t)plan.size());
    d.write(plan.data(), plan.size());
    if (!d)
        throw std::runtime_error("cannot write dump next to " + param.compressed_data_path);
}

int main(int argc, char *argv[]) { return asz_reference_s1_compress_main(argc, argv); }
