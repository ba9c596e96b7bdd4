#include "kcig_rsf.h"

#include <ctype.h>
#include <errno.h>
#include <limits.h>
#include <math.h>
#include <pwd.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include <fstream>
#include <sstream>
#include <vector>

#include "kcig_common.h"

namespace kcig {

long long RsfFile::count() const
{
    long long c = 1;
    for (int i = 0; i < (ndim > 0 ? ndim : 1); i++) c *= n[i];
    return c;
}

static std::string dir_of(const std::string &p)
{
    const size_t s = p.find_last_of('/');
    return s == std::string::npos ? std::string(".") : p.substr(0, s);
}

static std::string base_of(const std::string &p)
{
    const size_t s = p.find_last_of('/');
    return s == std::string::npos ? p : p.substr(s + 1);
}

static bool parse_int_str(const std::string &s, int *v)
{
    char *e = nullptr;
    long x = strtol(s.c_str(), &e, 10);
    if (e == s.c_str() || *e) return false;
    *v = (int)x;
    return true;
}

static bool parse_double_str(const std::string &s, double *v)
{
    char *e = nullptr;
    double x = strtod(s.c_str(), &e);
    if (e == s.c_str() || *e) return false;
    *v = x;
    return true;
}

// The SEP layer names a file by its absolute path (se_uri.cpp:67-150): a
// relative name is resolved against the working directory, "." components
// are dropped and ".." removes the component before it.
static std::string current_dir()
{
    char cwd[PATH_MAX] = ".";
    if (!getcwd(cwd, sizeof cwd)) strcpy(cwd, ".");
    return cwd;
}

static std::string sep_absolute(const std::string &path)
{
    std::vector<std::string> parts;
    auto add = [&parts](const std::string &p) {
        std::istringstream items(p);
        for (std::string item; std::getline(items, item, '/');) {
            if (item.empty() || item == ".") continue;
            if (item == "..") {
                if (!parts.empty()) parts.pop_back();
            } else {
                parts.push_back(item);
            }
        }
    };
    if (path.empty() || path[0] != '/') add(current_dir());
    add(path);
    std::string out = "/";
    for (size_t i = 0; i < parts.size(); i++) out += (i ? "/" : "") + parts[i];
    return out;
}

// se_fs_sep.cpp:740-745: the message of a header file that cannot be opened
static int sep_open_error(const std::string &path, int err)
{
    return set_error(KCIG_ERR_IO, "Cannot open SEP file '%s': current dir is %s, error code is %d - %s",
                     sep_absolute(path).c_str(), current_dir().c_str(), err, strerror(err));
}

int rsf_open(const std::string &path, RsfFile *f)
{
    *f = RsfFile();
    f->path = path;
    {
        FILE *probe = fopen(path.c_str(), "rb");
        if (!probe) return sep_open_error(path, errno);
        fclose(probe);
    }
    std::ifstream in(path, std::ios::binary);
    if (!in) return sep_open_error(path, errno ? errno : EIO);
    std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    const size_t eot = text.find('\x04');
    if (eot != std::string::npos) text.resize(eot);
    std::string in_name;
    std::istringstream lines(text);
    std::string line;
    while (std::getline(lines, line)) {
        const size_t h = line.find('#');
        if (h != std::string::npos) line.resize(h);
        size_t i = 0;
        while (i < line.size()) {
            while (i < line.size() && isspace((unsigned char)line[i])) i++;
            if (i >= line.size()) break;
            std::string tok;
            char q = 0;
            while (i < line.size() && (q || !isspace((unsigned char)line[i]))) {
                const char c = line[i++];
                if (q && c == q) { q = 0; continue; }
                if (!q && (c == '"' || c == '\'')) { q = c; continue; }
                tok.push_back(c);
            }
            const size_t eq = tok.find('=');
            if (eq == std::string::npos || eq == 0) continue;
            const std::string k = tok.substr(0, eq), v = tok.substr(eq + 1);
            int idx;
            if ((k[0] == 'n' || k[0] == 'o' || k[0] == 'd') && parse_int_str(k.substr(1), &idx) && idx >= 1 &&
                idx <= 9) {
                double dv;
                if (!parse_double_str(v, &dv)) continue;
                if (k[0] == 'n') {
                    if (dv < 1.0) continue;
                    f->n[idx - 1] = (int)dv;
                } else if (k[0] == 'o') {
                    f->o[idx - 1] = dv;
                } else {
                    if (dv == 0.0) continue;
                    f->d[idx - 1] = dv;
                }
                if (idx > f->ndim) f->ndim = idx;
                continue;
            }
            if (k == "in") {
                if (!v.empty()) in_name = v;
                continue;
            }
            if (k == "esize") {
                int e;
                if (parse_int_str(v, &e)) f->esize = e;
                continue;
            }
            if (k == "data_format") {
                if (v == "native_float") f->native = true;
                else if (v == "xdr_float") f->native = false;
                continue;
            }
            f->extra[k] = v;
        }
    }
    if (in_name.empty())
        return set_error(KCIG_ERR_IO, "Missing required SEP global header 'in' in file '%s'", path.c_str());
    if (in_name == "-" || in_name == "stdin")
        return set_error(KCIG_ERR_UNSUPPORTED, "inline SEP data (in=stdin) is not supported: '%s'", path.c_str());
    f->binary = in_name[0] == '/' ? in_name : dir_of(path) + "/" + in_name;
    if (f->esize != 4) return set_error(KCIG_ERR_IO, "Only esize=4 float data is supported: '%s'", path.c_str());
    return KCIG_OK;
}

int rsf_read(const RsfFile &f, long long offset, long long count, float *dst)
{
    FILE *fp = fopen(f.binary.c_str(), "rb");
    if (!fp) return set_error(KCIG_ERR_IO, "Cannot open data file '%s' of '%s'", f.binary.c_str(), f.path.c_str());
    if (fseeko(fp, (off_t)offset * 4, SEEK_SET) != 0) {
        fclose(fp);
        return set_error(KCIG_ERR_IO, "Failed to seek '%s'", f.binary.c_str());
    }
    const size_t got = fread(dst, 4, (size_t)count, fp);
    fclose(fp);
    if ((long long)got != count)
        return set_error(KCIG_ERR_IO, "Failed to read %lld floats from '%s' (file truncated)", count, f.binary.c_str());
    if (!f.native) {
        uint32_t *u = (uint32_t *)dst;
        for (long long i = 0; i < count; i++) u[i] = __builtin_bswap32(u[i]);
    }
    return KCIG_OK;
}

// _sep_print_a_double (se_fs_sep.cpp:67-93)
static std::string fmt_double(double v)
{
    char s[128];
    if (v == floor(v) && fabs(v) < 9.2e18) {
        snprintf(s, sizeof s, "%lld", (long long)v);
        return s;
    }
    snprintf(s, sizeof s, "%.12f", v);
    char *p = strrchr(s, '.');
    if (p) {
        char *z = nullptr;
        for (++p; *p; ++p) {
            if (*p == '0') { if (!z) z = p; }
            else z = nullptr;
        }
        if (z) *z = 0;
    }
    return s;
}

// the program named in the history line of the headers this process writes
static std::string g_program = "kirchmig2d_cig";

void rsf_set_program(const std::string &name) { g_program = name; }

int rsf_write(const std::string &path, int ndim, const int *n, const double *o, const double *d,
              const std::vector<std::pair<std::string, std::string>> &keys, const float *data, long long count)
{
    const std::string bin = path + "@";
    FILE *fb = fopen(bin.c_str(), "wb");
    if (!fb) return set_error(KCIG_ERR_IO, "Cannot open SEP file '%s'", bin.c_str());
    if (count > 0 && fwrite(data, 4, (size_t)count, fb) != (size_t)count) {
        fclose(fb);
        return set_error(KCIG_ERR_IO, "Failed to write '%s'", bin.c_str());
    }
    fclose(fb);
    FILE *fh = fopen(path.c_str(), "w");
    if (!fh) return sep_open_error(path, errno);
    char cwd[PATH_MAX] = ".";
    if (!getcwd(cwd, sizeof cwd)) strcpy(cwd, ".");
    char host[256] = "unknown_host";
    gethostname(host, sizeof host);
    const char *user = getenv("USER");
    if (!user) {
        struct passwd *pw = getpwuid(getuid());
        user = pw ? pw->pw_name : "unknown_user";
    }
    time_t t = time(nullptr);
    char tb[64];
    ctime_r(&t, tb);
    fprintf(fh, "\n%s\t\"%s\"\t%s@%s\t%s", g_program.c_str(), cwd, user, host, tb);
    fprintf(fh, "\tin=\"%s\"\n", base_of(bin).c_str());
    fprintf(fh, "\tdata_format=\"native_float\"\n");
    for (int i = 0; i < ndim; i++) fprintf(fh, "\tn%d=%d\n", i + 1, n[i]);
    for (int i = 0; i < ndim; i++) fprintf(fh, "\td%d=%s\n", i + 1, fmt_double(d[i]).c_str());
    for (int i = 0; i < ndim; i++) fprintf(fh, "\to%d=%s\n", i + 1, fmt_double(o[i]).c_str());
    fprintf(fh, "\tesize=4\n");
    for (auto &kv : keys) fprintf(fh, "\t%s=\"%s\"\n", kv.first.c_str(), kv.second.c_str());
    fclose(fh);
    return KCIG_OK;
}

}  // namespace kcig
