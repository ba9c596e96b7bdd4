// key=value / par=<file> parameter store with the lookup rules of the
// reference's se_par_init (SEFILESYSTEM/src/se_par_sep.cpp:185-340): argv
// tokens and par= files are read in order, a later key replaces an earlier
// one, quotes around a value are removed, '#' starts a comment in a file.
// Integers are read through a double and truncated (se_get_par_int32,
// :432-435); floats through a double (se_get_par_float, :442-445).
#pragma once

#include <map>
#include <string>

namespace kcig {

class ParMap {
   public:
    // Returns 0, or KCIG_ERR_IO when a par= file cannot be read.
    int parse(int argc, char **argv);
    int add_file(const std::string &path);
    void add_token(const std::string &tok);
    bool have(const char *k) const { return kv_.count(k) != 0; }
    const std::string &str(const char *k) const { return kv_.at(k); }
    // Returns 0 or KCIG_ERR_ARG when the value is not a number.
    int get_int(const char *k, int *v) const;
    int get_float(const char *k, float *v) const;

   private:
    std::map<std::string, std::string> kv_;
};

}  // namespace kcig
