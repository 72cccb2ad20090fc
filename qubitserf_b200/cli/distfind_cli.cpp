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
#include <iterator>
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

// Appends rows of one fixed width; the first row sets the width.  `where` names the
// source in error messages.
class RowSink {
public:
    explicit RowSink(std::string where) : where_(std::move(where)) {}
    void add(const std::vector<uint8_t>& row, int line) {
        if (m_.rows == 0) {
            m_.cols = (int)row.size();
            first_line_ = line;
        } else if ((int)row.size() != m_.cols) {
            die(where_ + ": line " + std::to_string(line) + " has " + std::to_string(row.size()) +
                " entries, line " + std::to_string(first_line_) + " has " +
                std::to_string(m_.cols));
        }
        m_.bits.insert(m_.bits.end(), row.begin(), row.end());
        ++m_.rows;
    }
    Matrix take() { return std::move(m_); }
    int rows() const { return m_.rows; }

private:
    std::string where_;
    Matrix m_;
    int first_line_ = 0;
};

// A 0/1 matrix file: one row per non-blank line, entries separated by blanks, each entry a
// single 0 or 1.
Matrix read_matrix_file(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) die(path + ": cannot be opened");
    const std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    RowSink sink(path);
    std::vector<uint8_t> row;
    int line = 1;
    size_t i = 0;
    while (i <= text.size()) {
        const char c = i < text.size() ? text[i] : '\n';
        if (c == '\n') {
            if (!row.empty()) sink.add(row, line);
            row.clear();
            ++line;
            ++i;
            continue;
        }
        if (std::isspace((unsigned char)c)) { ++i; continue; }
        size_t j = i;   // one entry: up to the next blank
        while (j < text.size() && !std::isspace((unsigned char)text[j])) ++j;
        const std::string entry = text.substr(i, j - i);
        if (entry != "0" && entry != "1")
            die(path + ": line " + std::to_string(line) + ": entry '" + entry + "' is not 0 or 1");
        row.push_back((uint8_t)(entry[0] - '0'));
        i = j;
    }
    if (sink.rows() == 0) die(path + ": no rows");
    return sink.take();
}

// Pauli letters: bit 0 = X part, bit 1 = Z part; 4 = not a Pauli letter.
struct PauliTable {
    uint8_t code[256];
    PauliTable() {
        std::fill(code, code + 256, (uint8_t)4);
        for (char c : std::string("I._ ")) code[(unsigned char)c] = 0;
        for (char c : std::string("Xx")) code[(unsigned char)c] = 1;
        for (char c : std::string("Zz")) code[(unsigned char)c] = 2;
        for (char c : std::string("Yy")) code[(unsigned char)c] = 3;
    }
};
const PauliTable kPauli;

// x and z parts of one Pauli string; `what` names it in error messages.
void decode_pauli(const std::string& s, const std::string& what, std::vector<uint8_t>& x,
                  std::vector<uint8_t>& z, int* kinds) {
    x.assign(s.size(), 0);
    z.assign(s.size(), 0);
    int seen = 0;
    for (size_t j = 0; j < s.size(); ++j) {
        const uint8_t c = kPauli.code[(unsigned char)s[j]];
        if (c == 4)
            die(what + ": character '" + std::string(1, s[j]) +
                "' is not a Pauli letter (I . _ X Z Y)");
        x[j] = c & 1u;
        z[j] = (c >> 1) & 1u;
        seen |= c;
    }
    if (kinds) *kinds = seen;
}

// Generator strings from stdin: one per line up to a blank line or the end of input.  Each
// must be a pure X or a pure Z string (CSS input); identity-only lines carry no generator.
void read_css_generators(Matrix& X, Matrix& Z, int& n, bool& any) {
    RowSink xs("input"), zs("input");
    std::string s;
    int line = 0;
    n = -1;
    any = false;
    std::vector<uint8_t> x, z;
    while (std::getline(std::cin, s)) {
        ++line;
        if (!s.empty() && s.back() == '\r') s.pop_back();
        if (s.empty()) break;
        any = true;
        if (n < 0) n = (int)s.size();
        if ((int)s.size() != n)
            die("input line " + std::to_string(line) + ": length " + std::to_string(s.size()) +
                ", the first line has " + std::to_string(n));
        int kinds = 0;
        decode_pauli(s, "input line " + std::to_string(line), x, z, &kinds);
        if (kinds == 3)
            die("input line " + std::to_string(line) +
                ": not a pure X or pure Z generator (CSS input only)");
        if (kinds == 1) xs.add(x, line);
        else if (kinds == 2) zs.add(z, line);
    }
    X = xs.take();
    Z = zs.take();
    X.cols = Z.cols = std::max(n, 0);
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
        Matrix Gx, Gz;
        int n = 0;
        bool any = false;
        read_css_generators(Gx, Gz, n, any);
        if (!any) die("operator mode: no generator lines on stdin");
        if ((int)o.op.size() != n)
            die("operator has length " + std::to_string(o.op.size()) + ", the generators " +
                std::to_string(n));
        std::vector<uint8_t> z, x;
        decode_pauli(o.op, "operator", x, z, nullptr);
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
        if (X.cols != Z.cols)
            die("--hx has " + std::to_string(X.cols) + " columns, --hz " + std::to_string(Z.cols));
    } else {
        int n = 0;
        bool any = false;
        read_css_generators(X, Z, n, any);
        if (!any) die("no generator lines on stdin (Pauli strings, or --hx/--hz files)");
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
