// Host side of the C ABI: errors, the .ini reader, the circuit.txt parser and
// the lowering of parsed gates to kernel ops.  Plain C++, no CUDA.
//
// The grammar, defaults and coefficient formulas follow the reference's MEM
// path; each function cites the reference code it stands in for.
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "qk_internal.h"

namespace qk {

static thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

void clear_error() { g_last_error.clear(); }

// ---------------------------------------------------------------------------
// .ini reader.  Same observable behaviour as the vendored inih + INIReader the
// reference uses (src/ini.h:97-119, src/INIReader.cpp:36-60): "[section]"
// headers, "name = value" or "name : value", ';' / '#' comment lines, ';'
// inline comments after whitespace, lower-cased section and key names,
// repeated keys joined with '\n', a leading UTF-8 BOM skipped.  Only a file
// that cannot be opened is an error (the reference checks ParseError() < 0
// only, src/simulator.cpp:190-193).
// ---------------------------------------------------------------------------
namespace {

std::string trim(const std::string &s) {
    size_t b = 0, e = s.size();
    while (b < e && std::isspace((unsigned char)s[b])) ++b;
    while (e > b && std::isspace((unsigned char)s[e - 1])) --e;
    return s.substr(b, e - b);
}

std::string lower(std::string s) {
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

struct Ini {
    std::map<std::string, std::string> values;  // "section=name" -> value

    bool load(const char *path) {
        std::ifstream f(path);
        if (!f) return false;
        std::string line, section, prev_key;
        bool first = true;
        while (std::getline(f, line)) {
            if (first && line.size() >= 3 && (unsigned char)line[0] == 0xEF &&
                (unsigned char)line[1] == 0xBB && (unsigned char)line[2] == 0xBF)
                line = line.substr(3);
            first = false;
            // continuation line: leading whitespace after a key (INI_ALLOW_MULTILINE)
            bool indented = !line.empty() && std::isspace((unsigned char)line[0]);
            std::string t = trim(line);
            if (t.empty() || t[0] == ';' || t[0] == '#') continue;
            // inline ';' comment preceded by whitespace (INI_INLINE_COMMENT_PREFIXES ";")
            for (size_t i = 1; i < t.size(); ++i)
                if (t[i] == ';' && std::isspace((unsigned char)t[i - 1])) {
                    t = trim(t.substr(0, i));
                    break;
                }
            if (indented && !prev_key.empty() && t[0] != '[') {
                values[prev_key] += "\n" + t;
                continue;
            }
            if (t[0] == '[') {
                size_t e = t.find(']');
                if (e != std::string::npos) section = lower(trim(t.substr(1, e - 1)));
                prev_key.clear();
                continue;
            }
            size_t eq = t.find_first_of("=:");
            if (eq == std::string::npos) continue;  // inih records an error line and goes on
            std::string key = section + "=" + lower(trim(t.substr(0, eq)));
            std::string val = trim(t.substr(eq + 1));
            auto it = values.find(key);
            if (it == values.end()) values[key] = val;
            else it->second += "\n" + val;
            prev_key = key;
        }
        return true;
    }
    std::string get(const char *section, const char *name, const char *dflt) const {
        auto it = values.find(lower(section) + "=" + lower(name));
        return it == values.end() ? std::string(dflt) : it->second;
    }
    long get_int(const char *section, const char *name, long dflt) const {
        std::string v = get(section, name, "");
        const char *s = v.c_str();
        char *end;
        long n = std::strtol(s, &end, 0);
        return end > s ? n : dflt;
    }
};

}  // namespace

// ---------------------------------------------------------------------------
// Gate lowering: the coefficient formulas of the reference's MEM gates.
// ---------------------------------------------------------------------------
static inline void setc(double *m, int k, double re, double im) {
    m[2 * k] = re;
    m[2 * k + 1] = im;
}

int lower_gate(const qk_gate &g, Op &op) {
    std::memset(&op, 0, sizeof op);
    op.nq = g.nq;
    for (int i = 0; i < g.nq && i < QK_MAX_TARGETS; ++i) op.q[i] = g.q[i];
    const double phi = g.param;
    switch (g.kind) {
    case QK_GATE_H: {
        // HGATE: a0' = c (a0 + a1), a1' = c (a0 - a1), c = 0.70710678118
        // (src/circuit.cpp:245-248; the truncated literal is kept on purpose)
        const double c = 0.70710678118;
        op.kind = OP_DENSE1;
        setc(op.m, 0, c, 0); setc(op.m, 1, c, 0); setc(op.m, 2, c, 0); setc(op.m, 3, -c, 0);
        return QK_OK;
    }
    case QK_GATE_X:  // XGATE (src/circuit.cpp:255-257)
        op.kind = OP_DENSE1;
        setc(op.m, 1, 1, 0); setc(op.m, 2, 1, 0);
        return QK_OK;
    case QK_GATE_Y:  // YGATE: a0' = -i a1, a1' = i a0 (src/circuit.cpp:263-265)
        op.kind = OP_DENSE1;
        setc(op.m, 1, 0, -1); setc(op.m, 2, 0, 1);
        return QK_OK;
    case QK_GATE_Z:  // ZGATE: a1 *= -1 (src/circuit.cpp:271-272)
        op.kind = OP_PHASE1;
        setc(op.m, 0, -1, 0);
        return QK_OK;
    case QK_GATE_P:  // Phase_Gate_MEM: phi(cos phi, sin phi) (src/circuit.cpp:2655)
        op.kind = OP_PHASE1;
        setc(op.m, 0, std::cos(phi), std::sin(phi));
        return QK_OK;
    case QK_GATE_U1:  // U1GATE, row-major coefficients (src/circuit.cpp:274-277)
        op.kind = OP_DENSE1;
        for (int k = 0; k < 8; ++k) op.m[k] = g.coeff[k];
        return QK_OK;
    case QK_GATE_RX: {  // RX_Gate_MEM (src/circuit.cpp:2706-2709), RXGATE (:287-290)
        op.kind = OP_DENSE1;
        const double c = std::cos(phi / 2), s = std::sin(-phi / 2);
        setc(op.m, 0, c, 0); setc(op.m, 1, 0, s); setc(op.m, 2, 0, s); setc(op.m, 3, c, 0);
        return QK_OK;
    }
    case QK_GATE_RY: {  // RY_Gate_MEM (src/circuit.cpp:2734-2737), RYGATE (:297-300)
        op.kind = OP_DENSE1;
        const double c = std::cos(phi / 2), s = std::sin(phi / 2);
        setc(op.m, 0, c, 0); setc(op.m, 1, -s, 0); setc(op.m, 2, s, 0); setc(op.m, 3, c, 0);
        return QK_OK;
    }
    case QK_GATE_RZ:  // RZ_Gate_MEM (src/circuit.cpp:2762-2765), RZGATE (:307-309)
        op.kind = OP_DIAG1;
        setc(op.m, 0, std::cos(-phi / 2), std::sin(-phi / 2));
        setc(op.m, 1, std::cos(phi / 2), std::sin(phi / 2));
        return QK_OK;
    case QK_GATE_U2: {
        // U2_Gate_MEM (src/circuit.cpp:2807-2819): the file matrix is in basis
        // |q0 q1> with q0 the most significant bit; the reference permutes it
        // to little-endian: coeff[i] = matrix[res],
        // res = (b2 << 3) | (b3 << 2) | (b0 << 1) | b1 with b_k = bit k of i.
        op.kind = OP_DENSE2;
        for (int i = 0; i < 16; ++i) {
            int b0 = i & 1, b1 = (i >> 1) & 1, b2 = (i >> 2) & 1, b3 = (i >> 3) & 1;
            int res = (b2 << 3) | (b3 << 2) | (b0 << 1) | b1;
            op.m[2 * i] = g.coeff[2 * res];
            op.m[2 * i + 1] = g.coeff[2 * res + 1];
        }
        // A matrix of exact 0 / 1 entries that is a CNOT or SWAP, or any
        // diagonal matrix, runs as that cheaper op.  The reference's dense
        // product with these entries gives the same amplitudes (up to the
        // sign of zeros).
        auto permutation = [&](const int (&row)[4]) {   // row[c]: row of column c's 1
            for (int r = 0; r < 4; ++r)
                for (int c = 0; c < 4; ++c)
                    if (op.m[2 * (4 * r + c)] != (row[c] == r ? 1.0 : 0.0) || op.m[2 * (4 * r + c) + 1] != 0.0)
                        return false;
            return true;
        };
        static const int cx0[4] = {0, 3, 2, 1}, cx1[4] = {0, 1, 3, 2}, swp[4] = {0, 2, 1, 3};
        bool diagonal = true;
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c)
                if (r != c && (op.m[2 * (4 * r + c)] != 0.0 || op.m[2 * (4 * r + c) + 1] != 0.0)) diagonal = false;
        if (permutation(cx0) || permutation(cx1)) {
            op.aux = permutation(cx0) ? 0 : 1;   // control q[aux], target q[1 - aux]
            op.kind = OP_CX;
        } else if (permutation(swp)) {
            op.kind = OP_SWAP2;
        } else if (diagonal) {
            double dm[8];
            for (int k = 0; k < 4; ++k) { dm[2 * k] = op.m[2 * (5 * k)]; dm[2 * k + 1] = op.m[2 * (5 * k) + 1]; }
            op.kind = OP_DIAG2;
            std::memcpy(op.m, dm, sizeof dm);
        }
        return QK_OK;
    }
    case QK_GATE_SWAP:  // SWAPGate: exchange |01> and |10> (src/circuit.cpp:351-355)
        op.kind = OP_SWAP2;
        return QK_OK;
    case QK_GATE_CP:  // CPhase_Gate_MEM: exp_iPhi = (cos phi, sin phi) (src/circuit.cpp:2947-2949)
        op.kind = OP_PHASE2;
        setc(op.m, 0, std::cos(phi), std::sin(phi));
        return QK_OK;
    case QK_GATE_RZZ: {  // RZZ_Gate_MEM (src/circuit.cpp:2988-2991), RZZGATE (:365-369)
        op.kind = OP_DIAG2;
        const double nr = std::cos(-phi / 2), ni = std::sin(-phi / 2);
        const double pr = std::cos(phi / 2), pi = std::sin(phi / 2);
        setc(op.m, 0, nr, ni); setc(op.m, 1, pr, pi); setc(op.m, 2, pr, pi); setc(op.m, 3, nr, ni);
        return QK_OK;
    }
    case QK_GATE_VSWAP:
    case QK_GATE_MPI_VSWAP:
        // VSWAP_1_1 is a SWAP with type VSWAP (src/circuit.cpp:2937-2940);
        // VSWAP_k_k swaps qubit q[i] with q[k+i] (VSWAP_2_2:
        // src/circuit.cpp:3457-3556, checked against SWAP(q0,q2) SWAP(q1,q3) by
        // src/correctness/gate_check_MEM.py:314-348).
        op.kind = g.nq == 2 ? OP_SWAP2 : OP_PERM;
        op.aux = 1;   // a VSWAP: planners may rename qubits instead
        return QK_OK;
    default:
        return fail(QK_ERR_PARSE, "unknown gate kind %d", g.kind);
    }
}

// U^dag of a lowered op (same kind).
void invert_op(Op &op) {
    auto conj = [&](int k) { op.m[2 * k + 1] = -op.m[2 * k + 1]; };
    switch (op.kind) {
    case OP_DENSE1:
    case OP_DENSE2: {
        const int d = op.kind == OP_DENSE1 ? 2 : 4;
        double m[32];
        for (int r = 0; r < d; ++r)
            for (int c = 0; c < d; ++c) {
                m[2 * (r * d + c)] = op.m[2 * (c * d + r)];
                m[2 * (r * d + c) + 1] = -op.m[2 * (c * d + r) + 1];
            }
        std::memcpy(op.m, m, sizeof(double) * 2 * d * d);
        break;
    }
    case OP_CDENSE1:   // each of the two 2x2 matrices
        for (int h = 0; h < 2; ++h) {
            double *a = op.m + 8 * h;
            const double m01r = a[2], m01i = a[3];
            a[1] = -a[1];
            a[7] = -a[7];
            a[2] = a[4];
            a[3] = -a[5];
            a[4] = m01r;
            a[5] = -m01i;
        }
        break;
    case OP_PHASE1: case OP_PHASE2: conj(0); break;
    case OP_DIAG1: conj(0); conj(1); break;
    case OP_DIAG2: for (int k = 0; k < 4; ++k) conj(k); break;
    default: break;  // SWAP2 and PERM are their own inverses
    }
}

}  // namespace qk

using namespace qk;

// ---------------------------------------------------------------------------
// Gate line parser: Simulator::setGate_MEM (src/simulator.cpp:542-597) with
// setGate_1/2, setGate_Phase, setUnitary, setGate_vswap (:259-356) and
// check_targ_in_N (:764-774).
// ---------------------------------------------------------------------------
namespace {

bool parse_int(const std::string &tok, int32_t &out) {
    if (tok.empty()) return false;
    const char *s = tok.c_str();
    char *end;
    errno = 0;
    long v = std::strtol(s, &end, 10);
    if (*end != '\0' || errno) return false;
    if (v < INT32_MIN || v > INT32_MAX) return false;
    out = (int32_t)v;
    return true;
}

bool parse_double(const std::string &tok, double &out) {
    if (tok.empty()) return false;
    const char *s = tok.c_str();
    char *end;
    out = std::strtod(s, &end);
    return *end == '\0';
}

struct GateSpec {
    const char *token;
    int kind;
    int ntargets;   // operands that are qubit ids
    int nangles;    // trailing angle
    int ncoeff;     // complex coefficients
};

const GateSpec kSpecs[] = {
    {"H", QK_GATE_H, 1, 0, 0},          {"X", QK_GATE_X, 1, 0, 0},
    {"Y", QK_GATE_Y, 1, 0, 0},          {"Z", QK_GATE_Z, 1, 0, 0},
    {"P", QK_GATE_P, 1, 1, 0},          {"RX", QK_GATE_RX, 1, 1, 0},
    {"RY", QK_GATE_RY, 1, 1, 0},        {"RZ", QK_GATE_RZ, 1, 1, 0},
    {"U1", QK_GATE_U1, 1, 0, 4},        {"U2", QK_GATE_U2, 2, 0, 16},
    {"SWAP", QK_GATE_SWAP, 2, 0, 0},    {"CP", QK_GATE_CP, 2, 1, 0},
    {"RZZ", QK_GATE_RZZ, 2, 1, 0},      {"VSWAP_1_1", QK_GATE_VSWAP, 2, 0, 0},
    {"VSWAP_2_2", QK_GATE_VSWAP, 4, 0, 0}, {"VSWAP_3_3", QK_GATE_VSWAP, 6, 0, 0},
    {"VSWAP_4_4", QK_GATE_VSWAP, 8, 0, 0}, {"VSWAP_6_6", QK_GATE_VSWAP, 12, 0, 0},
    {"MPI_VSWAP_1_1", QK_GATE_MPI_VSWAP, 2, 0, 0},
    {"MPI_VSWAP_2_2", QK_GATE_MPI_VSWAP, 4, 0, 0},
};

}  // namespace

extern "C" int qk_gate_parse_line(const char *line, int total_qbit, qk_gate *out) {
    if (!line || !out) return fail(QK_ERR_ARG, "null argument");
    std::istringstream ss{std::string(line)};
    std::vector<std::string> tok;
    for (std::string t; ss >> t;) tok.push_back(t);
    if (tok.empty()) return fail(QK_ERR_PARSE, "[setGate]: Not implemented yet. (empty line)");
    const GateSpec *spec = nullptr;
    for (const auto &s : kSpecs)
        if (tok[0] == s.token) { spec = &s; break; }
    if (!spec) return fail(QK_ERR_PARSE, "[setGate]: Not implemented yet. (gate '%s')", tok[0].c_str());
    const size_t need = 1 + spec->ntargets + spec->nangles + 2 * spec->ncoeff;
    if (tok.size() < need)
        return fail(QK_ERR_PARSE, "gate %s needs %zu operands, got %zu", spec->token, need - 1,
                    tok.size() - 1);
    qk_gate g;
    std::memset(&g, 0, sizeof g);
    g.kind = spec->kind;
    g.nq = spec->ntargets;
    size_t k = 1;
    for (int i = 0; i < spec->ntargets; ++i, ++k)
        if (!parse_int(tok[k], g.q[i]))
            return fail(QK_ERR_PARSE, "gate %s: bad qubit '%s'", spec->token, tok[k].c_str());
    if (spec->nangles && !parse_double(tok[k++], g.param))
        return fail(QK_ERR_PARSE, "gate %s: bad angle '%s'", spec->token, tok[k - 1].c_str());
    for (int i = 0; i < 2 * spec->ncoeff; ++i, ++k)
        if (!parse_double(tok[k], g.coeff[i]))
            return fail(QK_ERR_PARSE, "gate %s: bad coefficient '%s'", spec->token, tok[k].c_str());
    // check_targ_in_N (src/simulator.cpp:764-774)
    for (int i = 0; i < g.nq; ++i)
        if (g.q[i] < 0 || g.q[i] >= total_qbit)
            return fail(QK_ERR_QUBIT, "[setGate]: Qubit Index Error (qubit %d, total_qbit %d)", g.q[i],
                        total_qbit);
    // The reference's loop nests and bit_string (src/MEM_Runner.cpp:90-99)
    // assume ascending targets; U2 asserts it (src/circuit.cpp:2809).  VSWAP
    // targets only need to be distinct: the engine applies SWAP(q[i], q[k+i]).
    if (g.kind == QK_GATE_VSWAP || g.kind == QK_GATE_MPI_VSWAP) {
        for (int i = 0; i < g.nq; ++i)
            for (int j = i + 1; j < g.nq; ++j)
                if (g.q[i] == g.q[j])
                    return fail(QK_ERR_ORDER, "%s: qubit %d repeated", spec->token, g.q[i]);
    } else {
        for (int i = 1; i < g.nq; ++i)
            if (g.q[i] <= g.q[i - 1])
                return fail(QK_ERR_ORDER, "%s: targets must be strictly ascending (%d, %d)", spec->token,
                            g.q[i - 1], g.q[i]);
    }
    *out = g;
    clear_error();
    return QK_OK;
}

static int parse_stream(std::istream &in, int is_subcircuit, int total_qbit, qk_circuit **out) {
    auto *c = new qk_circuit();
    std::string line;
    int lineno = 0;
    auto bad = [&](int code) {
        std::string m = qk_last_error();
        delete c;
        return fail(code, "line %d: %s", lineno, m.c_str());
    };
    if (!is_subcircuit) {
        // setupCircuit_MEM: one gate per line (src/simulator.cpp:601-615)
        while (std::getline(in, line)) {
            ++lineno;
            qk_gate g;
            int rc = qk_gate_parse_line(line.c_str(), total_qbit, &g);
            if (rc) return bad(rc);
            c->gates.push_back(g);
            c->group_sizes.push_back(1);
        }
    } else {
        // setupSubCircuits_MEM: "<k>" then k gate lines (src/simulator.cpp:619-636)
        while (std::getline(in, line)) {
            ++lineno;
            int32_t k;
            std::istringstream ls(line);
            std::string tok;
            ls >> tok;
            if (!parse_int(tok, k) || k < 0) {
                fail(QK_ERR_PARSE, "expected a group size, got '%s'", line.c_str());
                return bad(QK_ERR_PARSE);
            }
            for (int32_t i = 0; i < k; ++i) {
                if (!std::getline(in, line)) {
                    fail(QK_ERR_PARSE, "group of %d gates ends after %d", k, i);
                    return bad(QK_ERR_PARSE);
                }
                ++lineno;
                qk_gate g;
                int rc = qk_gate_parse_line(line.c_str(), total_qbit, &g);
                if (rc) return bad(rc);
                c->gates.push_back(g);
            }
            c->group_sizes.push_back(k);
        }
    }
    *out = c;
    clear_error();
    return QK_OK;
}

extern "C" {

const char *qk_last_error(void) { return g_last_error.c_str(); }

int qk_abi_version(void) { return QK_ABI_VERSION; }

int qk_config_load(const char *ini_path, qk_config *out) {
    if (!ini_path || !out) return fail(QK_ERR_ARG, "null argument");
    Ini ini;
    if (!ini.load(ini_path)) return fail(QK_ERR_IO, "Error parsing config.ini! (cannot open %s)", ini_path);
    qk_config c;
    std::memset(&c, 0, sizeof c);
    const char *S = "system";
    // setSEG (src/simulator.cpp:88-100)
    c.total_qbit = (int32_t)ini.get_int(S, "total_qbit", 0);
    c.mpi_qbit = (int32_t)ini.get_int(S, "mpi_qbit", 0);
    c.file_qbit = (int32_t)ini.get_int(S, "file_qbit", 0);
    c.chunk_qbit = (int32_t)ini.get_int(S, "chunk_qbit", 0);
    // setENV (src/simulator.cpp:140-186)
    c.is_subcircuit = (int32_t)ini.get_int(S, "is_subcircuit", 1);
    c.MPI_buffe_size = (int32_t)ini.get_int(S, "MPI_buffe_size", 16);
    c.MPI_testing = (int32_t)ini.get_int(S, "MPI_testing", 0);
    std::snprintf(c.runner_type, sizeof c.runner_type, "%s", ini.get(S, "runner_type", "IO").c_str());
    std::snprintf(c.dump_file, sizeof c.dump_file, "%s", ini.get(S, "dump_file", "").c_str());
    // engine-only keys (ignored by the reference)
    std::string prec = lower(ini.get(S, "precision", "c128"));
    if (prec == "c128" || prec == "complex128") c.precision = QK_C128;
    else if (prec == "c64" || prec == "complex64") c.precision = QK_C64;
    else return fail(QK_ERR_ARG, "precision must be c128 or c64, got '%s'", prec.c_str());
    c.fuse_width = (int32_t)ini.get_int(S, "fuse_width", 0);
    c.dump_binary = lower(ini.get(S, "dump_format", "txt")) == "bin";
    std::snprintf(c.init_file, sizeof c.init_file, "%s", ini.get(S, "init_file", "").c_str());
    c.device_qbit = (int32_t)ini.get_int(S, "device_qbit", 0);
    if (c.device_qbit < 0 || c.device_qbit > c.total_qbit - c.mpi_qbit)
        return fail(QK_ERR_ARG, "device_qbit must be in [0, %d], got %d", c.total_qbit - c.mpi_qbit, c.device_qbit);
    // the reference's asserts (src/simulator.cpp:98-99, :152)
    const int n_local = c.total_qbit - c.mpi_qbit;
    if (c.chunk_qbit < 1) return fail(QK_ERR_ARG, "chunk_qbit must be >= 1 (got %d)", c.chunk_qbit);
    if (n_local < c.file_qbit + c.chunk_qbit)
        return fail(QK_ERR_ARG, "total_qbit - mpi_qbit (%d) < file_qbit + chunk_qbit (%d)", n_local,
                    c.file_qbit + c.chunk_qbit);
    if (c.MPI_buffe_size < 2) return fail(QK_ERR_ARG, "MPI_buffe_size must be >= 2");
    *out = c;
    clear_error();
    return QK_OK;
}

int qk_circuit_load(const char *path, int is_subcircuit, int total_qbit, qk_circuit **out) {
    if (!path || !out) return fail(QK_ERR_ARG, "null argument");
    std::ifstream f(path);
    if (!f) return fail(QK_ERR_IO, "cannot open circuit file %s", path);
    return parse_stream(f, is_subcircuit, total_qbit, out);
}

int qk_circuit_parse(const char *text, int is_subcircuit, int total_qbit, qk_circuit **out) {
    if (!text || !out) return fail(QK_ERR_ARG, "null argument");
    std::istringstream in{std::string(text)};
    return parse_stream(in, is_subcircuit, total_qbit, out);
}

size_t qk_circuit_num_gates(const qk_circuit *c) { return c ? c->gates.size() : 0; }
const qk_gate *qk_circuit_gates(const qk_circuit *c) { return c ? c->gates.data() : nullptr; }
size_t qk_circuit_num_groups(const qk_circuit *c) { return c ? c->group_sizes.size() : 0; }
const int32_t *qk_circuit_group_sizes(const qk_circuit *c) { return c ? c->group_sizes.data() : nullptr; }
void qk_circuit_destroy(qk_circuit *c) { delete c; }

int qk_gate_matrix(const qk_gate *g, double *out, int *dim) {
    if (!g || !out || !dim) return fail(QK_ERR_ARG, "null argument");
    Op op;
    int rc = lower_gate(*g, op);
    if (rc) return rc;
    const int nq = g->nq;
    const int d = 1 << nq;
    std::memset(out, 0, sizeof(double) * 2 * d * d);
    auto put = [&](int r, int c, double re, double im) {
        out[2 * (r * d + c)] = re;
        out[2 * (r * d + c) + 1] = im;
    };
    switch (op.kind) {
    case OP_DENSE1:
    case OP_DENSE2:
        for (int k = 0; k < d * d; ++k) put(k / d, k % d, op.m[2 * k], op.m[2 * k + 1]);
        break;
    case OP_PHASE1: put(0, 0, 1, 0); put(1, 1, op.m[0], op.m[1]); break;
    case OP_DIAG1: put(0, 0, op.m[0], op.m[1]); put(1, 1, op.m[2], op.m[3]); break;
    case OP_PHASE2:
        for (int k = 0; k < 3; ++k) put(k, k, 1, 0);
        put(3, 3, op.m[0], op.m[1]);
        break;
    case OP_DIAG2:
        for (int k = 0; k < 4; ++k) put(k, k, op.m[2 * k], op.m[2 * k + 1]);
        break;
    case OP_SWAP2: put(0, 0, 1, 0); put(1, 2, 1, 0); put(2, 1, 1, 0); put(3, 3, 1, 0); break;
    case OP_CX:
        if (op.aux == 0) { put(0, 0, 1, 0); put(3, 1, 1, 0); put(2, 2, 1, 0); put(1, 3, 1, 0); }
        else { put(0, 0, 1, 0); put(1, 1, 1, 0); put(3, 2, 1, 0); put(2, 3, 1, 0); }
        break;
    case OP_PERM: {
        const int k = nq / 2;
        for (int c = 0; c < d; ++c) {
            int r = c;
            for (int i = 0; i < k; ++i) {
                int a = (c >> i) & 1, b = (c >> (k + i)) & 1;
                r = (r & ~(1 << i) & ~(1 << (k + i))) | (b << i) | (a << (k + i));
            }
            put(r, c, 1, 0);
        }
        break;
    }
    }
    *dim = d;
    clear_error();
    return QK_OK;
}

}  // extern "C"
