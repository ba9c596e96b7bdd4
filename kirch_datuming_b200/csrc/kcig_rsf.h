// RSF/SEP subset of the reference's SEFILESYSTEM (src/se_fs_sep.cpp): text
// header of key=value tokens, FP32 binary named by in=, native or xdr floats.
#pragma once

#include <map>
#include <string>
#include <vector>

namespace kcig {

struct RsfFile {
    std::string path;        // header path
    std::string binary;      // resolved data path
    int ndim = 0;
    int n[9] = {0, 1, 1, 1, 1, 1, 1, 1, 1};
    double o[9] = {0}, d[9] = {1, 1, 1, 1, 1, 1, 1, 1, 1};
    int esize = 4;
    bool native = false;     // data_format="native_float" (default xdr, se_fs_sep.cpp:458)
    std::map<std::string, std::string> extra;
    long long count() const;
};

// Parse a header (se_fs_sep.cpp:440-700).  Returns 0 or KCIG_ERR_IO with the
// reference's message in kcig_last_error().
int rsf_open(const std::string &path, RsfFile *f);
// Read `count` floats starting at element `offset`.
int rsf_read(const RsfFile &f, long long offset, long long count, float *dst);
// The program name written in the history line of new headers (default
// kirchmig2d_cig); each drop-in tool sets its own.
void rsf_set_program(const std::string &name);
// Write a new native_float header + "<path>@" binary (se_fs_sep.cpp:704-977).
// keys are written after esize, in the given order.
int rsf_write(const std::string &path, int ndim, const int *n, const double *o, const double *d,
              const std::vector<std::pair<std::string, std::string>> &keys, const float *data, long long count);

}  // namespace kcig
