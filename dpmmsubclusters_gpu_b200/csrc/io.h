// io.h -- the two file formats the reference's CLI path reads: the --params_path JSON
// (jsoncpp with comments allowed, global_params.cpp:8-70) and the N x D .npy data file
// (cnpy, utils.cpp:12-57).  Small self-contained readers.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace dpmm {
namespace io {

struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0;
    std::string str;
    std::vector<Json> arr;
    std::map<std::string, Json> obj;

    bool is_null() const { return kind == Null; }
    const Json& operator[](const std::string& key) const;   // Null when absent
    const Json& operator[](size_t i) const;                  // Null when out of range
    size_t size() const { return kind == Array ? arr.size() : (kind == Object ? obj.size() : 0); }
    double as_double(double dflt) const;
    long long as_int(long long dflt) const;
    bool as_bool(bool dflt) const;
};

// Parses JSON text; `//` line and `/* */` block comments are skipped.  Returns false and
// sets err on malformed input.
bool parse_json(const std::string& text, Json& out, std::string& err);
bool read_file(const std::string& path, std::string& out);

// Reads a 2-D .npy array (C or Fortran order) of float64/float32/int8-64/uint8-64/bfloat16
// ('<V2' with descr bfloat16 or ml_dtypes' name) into point-major doubles: rows = points.
// Integer and bf16 data are converted exactly (unlike the reference's loader, which reads every
// 4-byte type as float and every 2-byte type as short, utils.cpp:26-50).
bool read_npy(const std::string& path, std::vector<double>& data, int64_t& rows, int64_t& cols, std::string& err);
// Writes a 2-D float64 / int32 C-order .npy.
bool write_npy_f64(const std::string& path, const double* data, int64_t rows, int64_t cols);
bool write_npy_i32(const std::string& path, const int32_t* data, int64_t rows, int64_t cols);

}  // namespace io
}  // namespace dpmm
