// Drop-in for the reference tool layercom_cig (src/layercom_cig.cpp): the
// same key=value arguments, RSF header rules, checks, messages and output
// header; the scaling and blending of every depth window run on the device
// (kcig_stitch_window), the full-depth volume stays there until it is written.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <regex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/kcig.h"

namespace {

namespace fs = std::filesystem;
using KeyVals = std::map<std::string, std::string>;

[[noreturn]] void stop(const std::string &msg) { throw std::runtime_error(msg); }

bool same_word(std::string a, std::string b)
{
    auto low = [](std::string &s) {
        for (char &c : s) c = (char)std::tolower((unsigned char)c);
    };
    low(a);
    low(b);
    return a == b;
}

void replace_every(std::string &s, const std::string &from, const std::string &to)
{
    for (size_t p = s.find(from); p != std::string::npos; p = s.find(from, p + to.size())) s.replace(p, from.size(), to);
}

// ------------------------------------------------------------- arguments --
// (:56-104) key=value only; later keys win; empty values count as absent for
// the required ones
KeyVals arguments(int argc, char **argv)
{
    KeyVals kv;
    for (int i = 1; i < argc; ++i) {
        const std::string s = argv[i];
        const size_t eq = s.find('=');
        if (eq == std::string::npos || eq == 0) stop("Arguments must use key=value form; bad argument: " + s);
        kv[s.substr(0, eq)] = s.substr(eq + 1);
    }
    return kv;
}

std::string required(const KeyVals &kv, const std::string &key)
{
    const auto it = kv.find(key);
    if (it == kv.end() || it->second.empty()) stop("Need " + key + "=");
    return it->second;
}

int int_arg(const KeyVals &kv, const std::string &key, int def)
{
    const auto it = kv.find(key);
    if (it == kv.end()) return def;
    size_t used = 0;
    long long v = 0;
    try {
        v = std::stoll(it->second, &used);
    } catch (...) {
        stop("Invalid integer " + key + "=" + it->second);
    }
    if (used != it->second.size() || v < std::numeric_limits<int>::min() || v > std::numeric_limits<int>::max())
        stop("Invalid integer " + key + "=" + it->second);
    return (int)v;
}

double real_arg(const KeyVals &kv, const std::string &key, double def)
{
    const auto it = kv.find(key);
    if (it == kv.end()) return def;
    size_t used = 0;
    double v = 0.0;
    try {
        v = std::stod(it->second, &used);
    } catch (...) {
        stop("Invalid number " + key + "=" + it->second);
    }
    if (used != it->second.size() || !std::isfinite(v)) stop("Invalid number " + key + "=" + it->second);
    return v;
}

// ----------------------------------------------------------- RSF headers --
// (:148-202) every key=value (or key="quoted value") of every line; n1 is
// required, n2/n3 default to 1; only native_float with esize=4; the binary is
// in= beside the header when such a file exists, else in= as written
struct Volume {
    fs::path header, binary;
    KeyVals kv;
    int n1 = 0, n2 = 1, n3 = 1;
    double o1 = 0.0, o2 = 0.0, o3 = 0.0, d1 = 1.0, d2 = 1.0, d3 = 1.0;
    std::string label1, label2, label3, unit1, unit2, unit3;
};

std::string unquote(const std::string &s)
{
    if (s.size() >= 2 && ((s.front() == '"' && s.back() == '"') || (s.front() == '\'' && s.back() == '\'')))
        return s.substr(1, s.size() - 2);
    return s;
}

int header_int(const KeyVals &kv, const std::string &key, int def, bool must)
{
    const auto it = kv.find(key);
    if (it == kv.end()) {
        if (must) stop("Missing RSF key " + key);
        return def;
    }
    size_t used = 0;
    int v = 0;
    try {
        v = std::stoi(it->second, &used);
    } catch (...) {
        stop("Invalid RSF integer " + key + "=" + it->second);
    }
    if (used != it->second.size()) stop("Invalid RSF integer " + key + "=" + it->second);
    return v;
}

double header_real(const KeyVals &kv, const std::string &key, double def)
{
    const auto it = kv.find(key);
    if (it == kv.end()) return def;
    size_t used = 0;
    double v = 0.0;
    try {
        v = std::stod(it->second, &used);
    } catch (...) {
        stop("Invalid RSF number " + key + "=" + it->second);
    }
    if (used != it->second.size() || !std::isfinite(v)) stop("Invalid RSF number " + key + "=" + it->second);
    return v;
}

std::string header_text(const KeyVals &kv, const std::string &key, const std::string &def)
{
    const auto it = kv.find(key);
    return it == kv.end() ? def : it->second;
}

Volume load_header(const fs::path &path)
{
    std::ifstream in(path);
    if (!in) stop("Cannot open RSF header: " + path.string());
    Volume v;
    v.header = path;
    static const std::regex pair_re(R"(([A-Za-z_][A-Za-z0-9_]*)\s*=\s*("[^"]*"|[^\s]+))");
    for (std::string line; std::getline(in, line);)
        for (std::sregex_iterator m(line.begin(), line.end(), pair_re), none; m != none; ++m)
            v.kv[(*m)[1].str()] = unquote((*m)[2].str());
    v.n1 = header_int(v.kv, "n1", 0, true);
    v.n2 = header_int(v.kv, "n2", 1, false);
    v.n3 = header_int(v.kv, "n3", 1, false);
    v.o1 = header_real(v.kv, "o1", 0.0);
    v.o2 = header_real(v.kv, "o2", 0.0);
    v.o3 = header_real(v.kv, "o3", 0.0);
    v.d1 = header_real(v.kv, "d1", 1.0);
    v.d2 = header_real(v.kv, "d2", 1.0);
    v.d3 = header_real(v.kv, "d3", 1.0);
    const int esize = header_int(v.kv, "esize", 4, false);
    const std::string format = header_text(v.kv, "data_format", "native_float");
    v.label1 = header_text(v.kv, "label1", "Depth");
    v.label2 = header_text(v.kv, "label2", "Lateral");
    v.label3 = header_text(v.kv, "label3", "Half-opening angle");
    v.unit1 = header_text(v.kv, "unit1", "");
    v.unit2 = header_text(v.kv, "unit2", "");
    v.unit3 = header_text(v.kv, "unit3", "degree");
    if (v.n1 <= 0 || v.n2 <= 0 || v.n3 <= 0) stop("Invalid RSF dimensions in " + path.string());
    if (esize != 4 || format != "native_float")
        stop("Only data_format=\"native_float\", esize=4 is supported: " + path.string());
    const std::string bin = header_text(v.kv, "in", "");
    if (bin.empty()) stop("Missing in= in RSF header: " + path.string());
    const fs::path p(bin);
    if (p.is_absolute()) {
        v.binary = p;
    } else {
        const fs::path beside = path.parent_path() / p;
        v.binary = fs::exists(beside) ? beside : p;
    }
    return v;
}

uint64_t samples(int n1, int n2, int n3)
{
    if (n1 <= 0 || n2 <= 0 || n3 <= 0) stop("Invalid nonpositive dimension");
    return (uint64_t)n1 * (uint64_t)n2 * (uint64_t)n3;
}

std::vector<float> load_samples(const Volume &v)
{
    const uint64_t count = samples(v.n1, v.n2, v.n3), bytes = count * sizeof(float);
    std::error_code ec;
    const auto have = fs::file_size(v.binary, ec);
    if (ec) stop("Cannot stat RSF binary: " + v.binary.string());
    if (have != bytes) {
        std::ostringstream m;  // paths stream quoted, as std::filesystem writes them
        m << "RSF binary size mismatch for " << v.header << ": expected " << bytes << " bytes, got " << have
          << " bytes from " << v.binary;
        stop(m.str());
    }
    if (count > (uint64_t)std::numeric_limits<size_t>::max()) stop("RSF volume too large: " + v.header.string());
    std::vector<float> data((size_t)count);
    std::ifstream in(v.binary, std::ios::binary);
    if (!in) stop("Cannot open RSF binary: " + v.binary.string());
    in.read(reinterpret_cast<char *>(data.data()), (std::streamsize)bytes);
    if (!in || (uint64_t)in.gcount() != bytes) stop("Short read from RSF binary: " + v.binary.string());
    return data;
}

// ----------------------------------------------------------- depth windows --
// (:245-304) one "start end [datum]" per line ('#' comments; ',', ';', tab
// and the full-width comma separate); START / END name the model's ends
struct Window {
    int start = 0, end = 0;
};

std::vector<Window> load_windows(const fs::path &file, int n1)
{
    std::ifstream in(file);
    if (!in) stop("Cannot open layer_txt=" + file.string());
    std::vector<Window> w;
    int line_no = 0;
    for (std::string line; std::getline(in, line);) {
        ++line_no;
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        replace_every(line, "\xEF\xBC\x8C", " ");
        for (char &c : line)
            if (c == ',' || c == ';' || c == '\t') c = ' ';
        std::istringstream words(line);
        std::vector<std::string> tok;
        for (std::string t; words >> t;) tok.push_back(t);
        if (tok.empty()) continue;
        const std::string at = std::to_string(line_no);
        if (tok.size() < 2) stop("layer_txt line " + at + " needs start,end");
        Window r;
        if (!same_word(tok[0], "START")) {
            try {
                r.start = std::stoi(tok[0]);
            } catch (...) {
                stop("Invalid layer start at line " + at);
            }
        }
        if (same_word(tok[1], "END")) {
            r.end = n1 - 1;
        } else {
            try {
                r.end = std::stoi(tok[1]);
            } catch (...) {
                stop("Invalid layer end at line " + at);
            }
            // the third column (datuming depth) is read and checked, not used
            if (tok.size() >= 3 && !same_word(tok[2], "END")) {
                try {
                    (void)std::stoi(tok[2]);
                } catch (...) {
                    stop("Invalid should_datum_abs at line " + at);
                }
            }
        }
        w.push_back(r);
    }
    if (w.empty()) stop("No layers found in " + file.string());
    if (w.front().start != 0) stop("First layer must start at depth sample 0");
    for (size_t i = 0; i < w.size(); ++i) {
        if (w[i].start < 0 || w[i].end < w[i].start || w[i].end >= n1)
            stop("Invalid layer range [" + std::to_string(w[i].start) + "," + std::to_string(w[i].end) + "]");
        if (i > 0 && w[i].start > w[i - 1].end)
            stop("Layer " + std::to_string(i + 1) + " does not overlap previous layer");
        if (i > 0 && w[i].end <= w[i - 1].end)
            stop("Layer " + std::to_string(i + 1) + " must extend deeper than previous layer");
    }
    if (w.back().end != n1 - 1) stop("Last layer must end at full-model sample " + std::to_string(n1 - 1));
    return w;
}

// (:306-329) one value for every window or one per window; ';' and the
// full-width comma also separate
std::vector<float> window_scales(std::string s, size_t n)
{
    std::vector<float> out(n, 1.0f);
    if (s.empty()) return out;
    replace_every(s, "\xEF\xBC\x8C", ",");
    std::replace(s.begin(), s.end(), ';', ',');
    std::vector<float> vals;
    std::stringstream items(s);
    for (std::string item; std::getline(items, item, ',');) {
        if (item.empty()) continue;
        size_t used = 0;
        float v = 0.0f;
        try {
            v = std::stof(item, &used);
        } catch (...) {
            stop("Invalid scale value: " + item);
        }
        while (used < item.size() && std::isspace((unsigned char)item[used])) ++used;
        if (used != item.size() || !std::isfinite(v)) stop("Invalid scale value: " + item);
        vals.push_back(v);
    }
    if (vals.size() == 1) std::fill(out.begin(), out.end(), vals[0]);
    else if (vals.size() == n) out = vals;
    else stop("scale= must contain 1 or " + std::to_string(n) + " values");
    return out;
}

bool same_axis(double a, double b) { return std::fabs(a - b) <= 1.0e-6 * std::max({1.0, std::fabs(a), std::fabs(b)}); }

// layer_image_base "x.rsf" -> "x_<k>.rsf", anything else -> "<name>_<k>"
fs::path window_file(const fs::path &base, int k)
{
    const std::string ext = base.extension().string();
    if (ext == ".rsf") return base.parent_path() / (base.stem().string() + "_" + std::to_string(k) + ext);
    return base.parent_path() / (base.filename().string() + "_" + std::to_string(k));
}

// (:350-410) binary at <header>@, the header's fields in the reference's
// order and precision, then both read back and checked
void write_volume(const fs::path &header, const Volume &first, const Volume &model, int n1, int n2, int n3,
                  const std::vector<float> &data)
{
    if (!header.parent_path().empty()) fs::create_directories(header.parent_path());
    const fs::path binary(header.string() + "@");
    {
        std::ofstream out(binary, std::ios::binary | std::ios::trunc);
        if (!out) stop("Cannot create output binary: " + binary.string());
        out.write(reinterpret_cast<const char *>(data.data()), (std::streamsize)(data.size() * sizeof(float)));
        if (!out) stop("Failed writing output binary: " + binary.string());
    }
    const uint64_t want = samples(n1, n2, n3) * sizeof(float);
    std::error_code ec;
    const uint64_t got = fs::file_size(binary, ec);
    if (ec || got != want) {
        std::ostringstream m;
        m << "Output binary size check failed: expected " << want << ", got " << (ec ? 0 : got);
        stop(m.str());
    }
    {
        std::ofstream h(header, std::ios::trunc);
        if (!h) stop("Cannot create output header: " + header.string());
        h << "in=\"" << binary.string() << "\"\n"
          << "data_format=\"native_float\"\n"
          << "esize=4\n"
          << "n1=" << n1 << "\n"
          << "n2=" << n2 << "\n"
          << "n3=" << n3 << "\n"
          << std::setprecision(12) << "o1=" << model.o1 << "\n"
          << "d1=" << model.d1 << "\n"
          << "o2=" << model.o2 << "\n"
          << "d2=" << model.d2 << "\n"
          << "o3=" << first.o3 << "\n"
          << "d3=" << first.d3 << "\n"
          << "label1=\"" << first.label1 << "\"\n"
          << "label2=\"" << first.label2 << "\"\n"
          << "label3=\"" << first.label3 << "\"\n";
        if (!first.unit1.empty()) h << "unit1=\"" << first.unit1 << "\"\n";
        if (!first.unit2.empty()) h << "unit2=\"" << first.unit2 << "\"\n";
        h << "unit3=\"" << (first.unit3.empty() ? "degree" : first.unit3) << "\"\n";
        if (!h) stop("Failed writing output header: " + header.string());
    }
    const Volume back = load_header(header);
    if (back.n1 != n1 || back.n2 != n2 || back.n3 != n3) stop("Output header dimension verification failed");
    const uint64_t back_bytes = samples(back.n1, back.n2, back.n3) * sizeof(float);
    if (fs::file_size(back.binary, ec) != back_bytes || ec) stop("Output RSF header/binary verification failed");
}

struct DeviceBuffer {
    float *p = nullptr;
    explicit DeviceBuffer(size_t n)
    {
        if (cudaMalloc(&p, n * sizeof(float)) != cudaSuccess) {
            p = nullptr;
            stop("cudaMalloc of " + std::to_string(n * sizeof(float)) + " bytes failed");
        }
    }
    ~DeviceBuffer() { cudaFree(p); }
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
};

void cuda_ok(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) stop(std::string(what) + ": " + cudaGetErrorString(e));
}

int run(int argc, char **argv)
{
    const KeyVals args = arguments(argc, argv);
    const fs::path model_file = required(args, "full_model");
    const fs::path base = required(args, "layer_image_base");
    const fs::path windows_file = required(args, "layer_txt");
    const fs::path output_file = required(args, "output_file");
    const int want_layers = int_arg(args, "nlayers", 0);
    const int want_angles = int_arg(args, "nangle", 0);
    const int stitch_blend = int_arg(args, "stitch_blend", 15);
    const int scalex_aper = int_arg(args, "scalex_aper", 0);
    const double scalex_scale = real_arg(args, "scalex_scale", 1.0);
    const auto sc = args.find("scale");
    const std::string scale_text = sc == args.end() ? "" : sc->second;
    if (stitch_blend < -1) stop("stitch_blend must be -1 or nonnegative");
    if (scalex_aper < 0) stop("scalex_aper must be nonnegative");
    if (!std::isfinite(scalex_scale)) stop("Invalid scalex_scale");

    const Volume model = load_header(model_file);
    const int n1 = model.n1, n2 = model.n2;
    const std::vector<Window> windows = load_windows(windows_file, n1);
    if (want_layers > 0 && want_layers != (int)windows.size()) stop("nlayers does not match layer_txt");
    const Volume first = load_header(window_file(base, 1));
    const int n3 = first.n3;
    if (want_angles > 0 && want_angles != n3) stop("nangle does not match first ADCIG n3");
    if (first.n2 != n2) stop("Lateral size mismatch between full_model and first ADCIG");
    if (!same_axis(first.o2, model.o2) || !same_axis(first.d2, model.d2))
        stop("Lateral axis mismatch between full_model and first ADCIG");
    std::cout << "INFO: CIG output dimensions: n1=" << n1 << " n2=" << n2 << " n3=" << n3 << "\n";
    std::cout << "INFO: Angle axis: o3=" << first.o3 << " d3=" << first.d3 << " n3=" << n3 << "\n";
    const std::vector<float> scales = window_scales(scale_text, windows.size());
    const uint64_t total = samples(n1, n2, n3);
    if (total > (uint64_t)std::numeric_limits<size_t>::max()) stop("Output CIG too large");

    DeviceBuffer out((size_t)total);
    cuda_ok(cudaMemset(out.p, 0, (size_t)total * sizeof(float)), "cudaMemset");
    int previous_end = -1;
    for (size_t k = 0; k < windows.size(); ++k) {
        const fs::path file = window_file(base, (int)k + 1);
        const Volume img = load_header(file);
        const int start = windows[k].start, end = windows[k].end, n1w = end - start + 1;
        if (img.n1 != n1w || img.n2 != n2 || img.n3 != n3) {
            std::ostringstream m;
            m << file << " dimensions are " << img.n1 << "," << img.n2 << "," << img.n3 << "; expected " << n1w
              << "," << n2 << "," << n3;
            stop(m.str());
        }
        if (!same_axis(img.o2, first.o2) || !same_axis(img.d2, first.d2) || !same_axis(img.o3, first.o3) ||
            !same_axis(img.d3, first.d3))
            stop("Lateral or angle axis mismatch in " + file.string());
        int overlap = 0;
        if (k > 0) {
            overlap = previous_end - start + 1;
            if (overlap <= 0) stop("No overlap for layer " + std::to_string(k + 1));
        }
        const int blend = (overlap > 0 && stitch_blend >= 0) ? std::min(stitch_blend, overlap) : overlap;
        std::cout << "INFO: Layer " << (k + 1) << ": " << file.string() << ", range=[" << start << "," << end
                  << "]" << ", overlap=" << overlap << ", keep_upper=" << overlap - blend << ", blend=" << blend
                  << ", scale=" << scales[k] << "\n";
        const std::vector<float> host = load_samples(img);
        DeviceBuffer win(host.size());
        cuda_ok(cudaMemcpy(win.p, host.data(), host.size() * sizeof(float), cudaMemcpyHostToDevice), "cudaMemcpy");
        long long nonfinite = 0;
        if (kcig_stitch_window(out.p, n1, n2, n3, win.p, start, end, previous_end, stitch_blend, scales[k],
                               k > 0 ? 1 : 0, scalex_aper, scalex_scale, &nonfinite, nullptr) != KCIG_OK)
            stop(kcig_last_error());
        if (nonfinite > 0) stop(file.string() + " contains non-finite samples after scaling");
        previous_end = end;
    }
    std::vector<float> result((size_t)total);
    cuda_ok(cudaMemcpy(result.data(), out.p, (size_t)total * sizeof(float), cudaMemcpyDeviceToHost), "cudaMemcpy");
    write_volume(output_file, first, model, n1, n2, n3, result);
    std::cout << "INFO: Finished CIG stitching: " << output_file.string() << "\n";
    std::cout << "INFO: Output binary: " << output_file.string() << "@\n";
    std::cout << "INFO: Output samples: " << total << ", bytes=" << total * sizeof(float) << "\n";
    return 0;
}

}  // namespace

extern "C" int kcig_run_layercom_cig_cli(int argc, char **argv)
{
    try {
        run(argc, argv);
        return KCIG_OK;
    } catch (const std::exception &e) {
        std::cerr << "ERROR: " << e.what() << "\n";
        return KCIG_ERR_ARG;
    }
}
