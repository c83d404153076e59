/* A stand-in for the two csv_tools functions that the reference's prediction sweep calls.
 *
 * Test infrastructure only. c_codes/s2_many_prediction.cpp:22 includes
 * "../third_party/csv_tools/c_codes/csv.hpp", but the csv_tools submodule is not checked out, so
 * the oracle build points that include at this file. Its format is not the csv_tools one (which is
 * not available): every write_csv_item call appends one line
 *
 *     <key0>;<key1>;...|<column>|<value>
 *
 * with doubles printed as %.17g, and create_csv_header writes "#" followed by the key names. The
 * golden-fixture script parses these lines; they carry every value the sweep computes at full
 * precision (its stdout prints them with %f).
 */
#ifndef ASZ_ORACLE_CSV_SHIM_H
#define ASZ_ORACLE_CSV_SHIM_H
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

namespace csv_tools {

inline void csv_shim_append(const std::string &path, const std::string &line) {
    FILE *f = std::fopen(path.c_str(), "a");
    if (!f) throw std::runtime_error("csv shim: cannot open " + path);
    std::fputs(line.c_str(), f);
    std::fputc('\n', f);
    std::fclose(f);
}

inline std::string csv_shim_num(double v) {
    char b[64];
    std::snprintf(b, sizeof b, "%.17g", v);
    return b;
}

template <class... Names>
void create_csv_header(const std::string &path, const Names &...names) {
    std::string line = "#";
    ((line += std::string(names) + ";"), ...);
    csv_shim_append(path, line);
}

inline std::string csv_shim_key(const std::vector<double> &key) {
    std::string s;
    for (size_t i = 0; i < key.size(); i++) s += (i ? ";" : "") + csv_shim_num(key[i]);
    return s;
}

inline void write_csv_item(const std::string &path, const std::vector<double> &key, const std::string &column, double v) {
    csv_shim_append(path, csv_shim_key(key) + "|" + column + "|" + csv_shim_num(v));
}

inline void write_csv_item(const std::string &path, const std::vector<double> &key, const std::string &column,
                           const std::string &v) {
    csv_shim_append(path, csv_shim_key(key) + "|" + column + "|" + v);
}

}  // namespace csv_tools
#endif
