// qsfb-distfind: the reference's distfind command line (cpp/distfind/cli/distfind_cli.cpp)
// over libqsfb200.so's C ABI.  Same flags, inputs and output: Pauli strings on stdin (one
// per line, I . _ identity, X / Z; a blank line or EOF ends the input; CSS only), or 0/1
// text matrices with --hx/--hz; stdout is just the number(s), unproven results and
// diagnostics go to stderr, usage errors exit 2.
//
//   --bz (default) | --mitm | --cc     method (cc: rc 5 where the reference runs its
//                                      connected-cluster solver)
//   --gpu | --cpu                      backend (default auto; there is no CPU path here)
//   --z | --x | --zx                   one side, or "<dZ> <dX>" (both sides to their own
//                                      proofs, as the reference's uncapped interleave)
//   --subsystem                        the X/Z rows are gauge generators (dressed distance)
//   -o/--operator PAULI                operator weight of PAULI modulo the generators read
//                                      from stdin (max(z, x); --zx: "<z> <x>")
//   --threads N, -v/--verbose, -h/--help
#include <algorithm>
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "qsf_b200.h"

namespace {

const char* kUsage =
    "Usage: qsfb-distfind [OPTIONS]\n"
    "       cat code.txt | qsfb-distfind [OPTIONS]\n"
    "       qsfb-distfind --hx Hx.txt --hz Hz.txt [OPTIONS]\n"
    "\n"
    "Minimum distance of a CSS code on the GPU (libqsfb200.so).\n"
    "\n"
    "Input (default): Pauli stabiliser strings on stdin, one per line: I . _ identity,\n"
    "X and Z; a blank line or EOF ends the input.  Every row is pure X- or pure Z-type.\n"
    "\n"
    "Method:    --bz (default)  --mitm  --cc\n"
    "Backend:   --gpu  --cpu    (default: auto; this build runs on the GPU only)\n"
    "Output:    default = minimum distance; --zx = \"<dZ> <dX>\"; --z / --x = one value\n"
    "Subsystem: --subsystem  the X/Z rows are gauge generators (dressed distance)\n"
    "Operator:  -o/--operator PAULI  weight of PAULI (may contain Y) modulo the generators\n"
    "           on stdin (default max(z,x); --zx = \"<z> <x>\")\n"
    "Other:     --threads N  --hx FILE  --hz FILE  -v/--verbose  -h/--help\n";

struct Options {
    std::string method = "bz", backend = "auto";
    char which = 'M';
    bool zx = false, subsystem = false, op_mode = false, verbose = false;
    std::string op, hx_path, hz_path;
    int threads = 0;
};

struct Matrix {
    int rows = 0, cols = 0;
    std::vector<uint8_t> bits;   // rows x cols, 0/1
};

[[noreturn]] void die(const std::string& msg) {
    std::cerr << "qsfb-distfind: " << msg << "\n";
    std::exit(2);
}

Matrix read_matrix_file(const std::string& path) {
    std::ifstream in(path);
    if (!in) die("cannot open file: " + path);
    Matrix m;
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::vector<uint8_t> row;
        std::string tok;
        while (ls >> tok) {
            if (tok == "0") row.push_back(0);
            else if (tok == "1") row.push_back(1);
            else die("matrix file " + path + " contains non-binary token '" + tok + "'");
        }
        if (row.empty()) continue;
        if (m.rows == 0) m.cols = (int)row.size();
        else if ((int)row.size() != m.cols) die("ragged matrix in " + path + " (rows have differing widths)");
        m.bits.insert(m.bits.end(), row.begin(), row.end());
        ++m.rows;
    }
    if (m.rows == 0) die("matrix file " + path + " is empty");
    return m;
}

std::vector<std::string> read_lines() {
    std::vector<std::string> lines;
    std::string line;
    while (std::getline(std::cin, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.empty()) break;
        lines.push_back(line);
    }
    return lines;
}

// X-type and Z-type rows of CSS generator strings ("what" names them in errors).
void split_css_rows(const std::vector<std::string>& lines, const char* what, Matrix& X,
                    Matrix& Z, int& n) {
    n = (int)lines[0].size();
    X.cols = Z.cols = n;
    for (size_t li = 0; li < lines.size(); ++li) {
        const std::string& s = lines[li];
        if ((int)s.size() != n) die(std::string(what) + "s have differing lengths");
        std::vector<uint8_t> x(n, 0), z(n, 0);
        bool hx = false, hz = false;
        for (int j = 0; j < n; ++j) {
            switch (s[j]) {
                case 'I': case '.': case '_': case ' ': break;
                case 'X': case 'x': x[j] = 1; hx = true; break;
                case 'Z': case 'z': z[j] = 1; hz = true; break;
                case 'Y': case 'y':
                    die(std::string(what) + " " + std::to_string(li + 1) +
                        " contains a Y -- only CSS codes are supported");
                default:
                    die(std::string(what) + " " + std::to_string(li + 1) +
                        " has an unrecognised character '" + s[j] + "'");
            }
        }
        if (hx && hz)
            die(std::string(what) + " " + std::to_string(li + 1) +
                " mixes X and Z -- only CSS codes are supported");
        if (hx) { X.bits.insert(X.bits.end(), x.begin(), x.end()); ++X.rows; }
        else if (hz) { Z.bits.insert(Z.bits.end(), z.begin(), z.end()); ++Z.rows; }
    }
}

const uint8_t* data_or_dummy(const Matrix& m) {
    static const uint8_t zero = 0;
    return m.bits.empty() ? &zero : m.bits.data();
}

DistfindResult distance(const Matrix& X, const Matrix& Z, char which, const Options& o) {
    DistfindResult r{};
    const int rc = o.subsystem
        ? distfind_subsystem_distance(data_or_dummy(X), X.rows, X.cols, data_or_dummy(Z), Z.rows,
                                      Z.cols, o.method.c_str(), which, o.backend.c_str(),
                                      o.threads, o.verbose ? 1 : 0, &r)
        : distfind_css_distance(data_or_dummy(X), X.rows, X.cols, data_or_dummy(Z), Z.rows,
                                Z.cols, o.method.c_str(), which, o.backend.c_str(), o.threads,
                                o.verbose ? 1 : 0, &r);
    if (rc != 0) {
        std::cerr << "qsfb-distfind: distance call failed (rc=" << rc << ")\n";
        std::exit(1);
    }
    return r;
}

void note_if_unproven(const DistfindResult& r, const char* label) {
    if (!r.proven)
        std::cerr << "qsfb-distfind: " << label << " d in [" << r.lower_bound << ", "
                  << r.distance << "] (not proven)\n";
}

int parse_count(const std::string& flag, const std::string& v) {
    if (v.empty() || !std::all_of(v.begin(), v.end(), [](unsigned char c) { return std::isdigit(c); }))
        die(flag + " expects a non-negative integer, got '" + v + "'");
    return std::atoi(v.c_str());
}

}  // namespace

int main(int argc, char** argv) {
    Options o;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto value = [&](const std::string& flag) -> std::string {
            if (i + 1 >= argc) die(flag + " requires a value");
            return argv[++i];
        };
        if (a == "-h" || a == "--help") { std::cout << kUsage; return 0; }
        else if (a == "--bz") o.method = "bz";
        else if (a == "--cc") o.method = "cc";
        else if (a == "--mitm") o.method = "mitm";
        else if (a == "--cpu") o.backend = "cpu";
        else if (a == "--gpu") o.backend = "gpu";
        else if (a == "--zx") o.zx = true;
        else if (a == "--z") o.which = 'Z';
        else if (a == "--x") o.which = 'X';
        else if (a == "--subsystem") o.subsystem = true;
        else if (a == "-o" || a == "--operator") { o.op_mode = true; o.op = value(a); }
        else if (a == "--threads") o.threads = parse_count(a, value(a));
        else if (a == "-v" || a == "--verbose") o.verbose = true;
        else if (a == "--hx") o.hx_path = value(a);
        else if (a == "--hz") o.hz_path = value(a);
        else die("unrecognised argument '" + a + "' (try --help)");
    }
    if (o.zx && o.which != 'M') die("--zx cannot be combined with --z or --x");
    if (o.hx_path.empty() != o.hz_path.empty()) die("--hx and --hz must be given together");

    if (o.op_mode) {
        if (!o.hx_path.empty())
            die("-o/--operator reads generators and the operator from stdin (no --hx/--hz)");
        const std::vector<std::string> lines = read_lines();
        if (lines.empty()) die("operator mode needs at least one generator line on stdin");
        Matrix Gx, Gz;
        int n = 0;
        split_css_rows(lines, "generator", Gx, Gz, n);
        if ((int)o.op.size() != n)
            die("operator length (" + std::to_string(o.op.size()) +
                ") differs from the generators (" + std::to_string(n) + ")");
        std::vector<uint8_t> z(n, 0), x(n, 0);
        for (int j = 0; j < n; ++j) {
            switch (o.op[j]) {
                case 'I': case '.': case '_': case ' ': break;
                case 'X': case 'x': x[j] = 1; break;
                case 'Z': case 'z': z[j] = 1; break;
                case 'Y': case 'y': x[j] = z[j] = 1; break;
                default: die(std::string("operator has an unrecognised character '") + o.op[j] + "'");
            }
        }
        // with --subsystem the generators are the gauge group: the coset is taken modulo it
        DistfindOpResult w{};
        const int rc = distfind_operator_weight(data_or_dummy(Gx), Gx.rows, n, data_or_dummy(Gz),
                                                Gz.rows, n, z.data(), x.data(), n, o.method.c_str(),
                                                o.backend.c_str(), o.threads, o.verbose ? 1 : 0, &w);
        if (rc != 0) {
            std::cerr << "qsfb-distfind: operator weight failed (rc=" << rc << ")\n";
            return 1;
        }
        if (!w.proven)
            std::cerr << "qsfb-distfind: operator weight not proven (z=" << w.z_weight
                      << ", x=" << w.x_weight << ")\n";
        if (o.zx) std::cout << w.z_weight << ' ' << w.x_weight << std::endl;
        else std::cout << std::max(w.z_weight, w.x_weight) << std::endl;
        return 0;
    }

    Matrix X, Z;
    if (!o.hx_path.empty()) {
        X = read_matrix_file(o.hx_path);
        Z = read_matrix_file(o.hz_path);
        if (X.cols != Z.cols) die("Hx and Hz have differing column counts (different number of qubits)");
    } else {
        const std::vector<std::string> lines = read_lines();
        if (lines.empty()) die("no stabilisers on stdin (provide Pauli strings or --hx/--hz)");
        int n = 0;
        split_css_rows(lines, "stabiliser", X, Z, n);
    }
    if (o.verbose)
        std::cerr << "qsfb-distfind: method=" << o.method << " backend=" << o.backend
                  << " qubits=" << X.cols << " Hx_rows=" << X.rows << " Hz_rows=" << Z.rows
                  << " device=" << qsfb_device_name() << "\n";
    if (o.zx) {
        const DistfindResult rz = distance(X, Z, 'Z', o), rx = distance(X, Z, 'X', o);
        note_if_unproven(rz, "dZ:");
        note_if_unproven(rx, "dX:");
        std::cout << rz.distance << ' ' << rx.distance << std::endl;
    } else {
        const DistfindResult r = distance(X, Z, o.which, o);
        note_if_unproven(r, o.which == 'Z' ? "dZ:" : o.which == 'X' ? "dX:" : "d:");
        std::cout << r.distance << std::endl;
    }
    return 0;
}
