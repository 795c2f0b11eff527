// Readers for the reference's input files, so that its example inputs drive this library
// without libconfig:
//   .ucf unit-cell file        geom::readGlobalGeom (src/geom_glob.cpp:190-295)
//   .exch exchange file        exch::get_exch_unitcell (src/exch_determine_exchange_matrix.cpp:27-144),
//                              libconfig syntax, parsed here by a small recursive-descent reader
//   csr_exch_mat.dat           read: src/exch.cpp:63-133; written: src/exch_unitcell.cpp:36-63
// All entry points are plain C; errors come back as ASD_E* codes with a message in `err`.
#include "../../include/asd.h"
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace {

struct ReadFail {
    int code;
    std::string msg;
};

void put_err(char* err, size_t len, const std::string& m) {
    if (err && len) std::snprintf(err, len, "%s", m.c_str());
}

// ---- libconfig subset: settings `name = value;` / `name : value;`, groups `{...}`, arrays
// `[...]` and lists `(...)` of scalars, strings, integers, floats, booleans; comments `#`,
// `//` and `/* */`.  Values are kept as text; groups nest by dotted path.
class Cfg {
public:
    explicit Cfg(const std::string& text) : s_(text) {}

    void parse() {
        settings("");
        skip();
        if (p_ != s_.size()) fail("unexpected text");
    }
    bool has(const std::string& k) const { return scalars_.count(k) || arrays_.count(k) || groups_.count(k); }
    bool has_group(const std::string& k) const { return groups_.count(k) != 0; }
    bool scalar(const std::string& k, std::string* v) const {
        auto it = scalars_.find(k);
        if (it == scalars_.end()) return false;
        *v = it->second;
        return true;
    }
    bool array(const std::string& k, std::vector<std::string>* v) const {
        auto it = arrays_.find(k);
        if (it == arrays_.end()) return false;
        *v = it->second;
        return true;
    }

private:
    const std::string s_;
    size_t p_ = 0;
    int line_ = 1;
    std::map<std::string, std::string> scalars_;
    std::map<std::string, std::vector<std::string>> arrays_;
    std::map<std::string, int> groups_;

    [[noreturn]] void fail(const std::string& m) const {
        throw ReadFail{ASD_EINVAL, "exchange file line " + std::to_string(line_) + ": " + m};
    }
    void skip() {
        for (;;) {
            while (p_ < s_.size() && std::isspace((unsigned char)s_[p_])) { if (s_[p_] == '\n') line_++; p_++; }
            if (p_ < s_.size() && s_[p_] == '#') { while (p_ < s_.size() && s_[p_] != '\n') p_++; continue; }
            if (p_ + 1 < s_.size() && s_[p_] == '/' && s_[p_ + 1] == '/') { while (p_ < s_.size() && s_[p_] != '\n') p_++; continue; }
            if (p_ + 1 < s_.size() && s_[p_] == '/' && s_[p_ + 1] == '*') {
                const size_t e = s_.find("*/", p_ + 2);
                if (e == std::string::npos) fail("unterminated comment");
                for (size_t q = p_; q < e; q++) if (s_[q] == '\n') line_++;
                p_ = e + 2;
                continue;
            }
            return;
        }
    }
    bool peek(char c) { skip(); return p_ < s_.size() && s_[p_] == c; }
    void expect(char c) {
        if (!peek(c)) fail(std::string("expected '") + c + "'");
        p_++;
    }
    std::string name() {
        skip();
        const size_t b = p_;
        if (p_ < s_.size() && (std::isalpha((unsigned char)s_[p_]) || s_[p_] == '*'))
            while (p_ < s_.size() && (std::isalnum((unsigned char)s_[p_]) || s_[p_] == '_' || s_[p_] == '-' || s_[p_] == '*')) p_++;
        if (p_ == b) fail("expected a setting name");
        return s_.substr(b, p_ - b);
    }
    std::string scalar_text() {
        skip();
        if (p_ < s_.size() && s_[p_] == '"') {
            std::string out;
            for (;;) {   // adjacent string literals concatenate
                p_++;
                while (p_ < s_.size() && s_[p_] != '"') {
                    if (s_[p_] == '\\' && p_ + 1 < s_.size()) p_++;
                    out += s_[p_++];
                }
                if (p_ >= s_.size()) fail("unterminated string");
                p_++;
                if (!peek('"')) break;
            }
            return out;
        }
        const size_t b = p_;
        while (p_ < s_.size() && (std::isalnum((unsigned char)s_[p_]) || std::strchr("+-._", s_[p_]))) p_++;
        if (p_ == b) fail("expected a value");
        return s_.substr(b, p_ - b);
    }
    void value(const std::string& key) {
        skip();
        if (peek('{')) {
            p_++;
            groups_[key] = 1;
            settings(key + ".");
            expect('}');
        } else if (peek('[') || peek('(')) {
            const char close = s_[p_] == '[' ? ']' : ')';
            p_++;
            std::vector<std::string> v;
            if (!peek(close)) {
                for (;;) {
                    if (peek('{') || peek('[') || peek('(')) fail("nested aggregates are not supported in " + key);
                    v.push_back(scalar_text());
                    if (peek(',')) { p_++; continue; }
                    break;
                }
            }
            expect(close);
            arrays_[key] = v;
        } else {
            scalars_[key] = scalar_text();
        }
    }
    void settings(const std::string& prefix) {
        for (;;) {
            skip();
            if (p_ >= s_.size() || s_[p_] == '}') return;
            const std::string k = prefix + name();
            skip();
            if (p_ < s_.size() && (s_[p_] == '=' || s_[p_] == ':')) p_++;
            else fail("expected '=' or ':' after " + k);
            value(k);
            skip();
            if (p_ < s_.size() && (s_[p_] == ';' || s_[p_] == ',')) p_++;
        }
    }
};

double to_double(const std::string& t, const std::string& what) {
    char* end = nullptr;
    const double v = std::strtod(t.c_str(), &end);
    if (end == t.c_str() || *end != '\0') throw ReadFail{ASD_EINVAL, "not a number in " + what + ": " + t};
    return v;
}

// Conversion to joules of the exchange units the reference accepts
// (src/exch_determine_exchange_matrix.cpp:103-126).
double unit_factor(const std::string& u) {
    if (u == "J" || u == "Joules" || u == "joules") return 1.0;
    if (u == "mRy") return 2.179872172e-18 * 1.0e-3;
    if (u == "eV") return 1.602176565e-19;
    if (u == "meV") return 1.602176565e-22;
    if (u == "Ry") return 2.179872172e-18;
    throw ReadFail{ASD_EINVAL, "Units of exchange energy not recognised: " + u};
}

// Neighbour cell offset as src/exch_unitcell.cpp:303-327 forms it: round half away from zero.
int32_t round_offset(double x) { return x < 0 ? (int32_t)(x - 0.5) : (int32_t)(x + 0.5); }

}  // namespace

extern "C" {

int asd_read_ucf(const char* path, int mesh_points, uint32_t* nms_out, uint32_t* nauc_out, asd_ucf_atom* atoms,
                 uint32_t cap, char* err, size_t err_len) {
    try {
        if (!path || !nms_out || !nauc_out) throw ReadFail{ASD_EINVAL, "path, nms and nauc are required"};
        std::ifstream in(path);
        if (!in) throw ReadFail{ASD_EINVAL, std::string("Could not open unit cell file ") + path};
        long long nms = -1, nauc = -1;
        in >> nms >> nauc;
        if (!in || nms < 1) throw ReadFail{ASD_EINVAL, "Could not read the number of magnetic species"};
        if (nauc < 1) throw ReadFail{ASD_EINVAL, "There are no atoms in the unit cell, check your unit cell file."};
        *nms_out = (uint32_t)nms;
        *nauc_out = (uint32_t)nauc;
        if (!atoms) return ASD_OK;
        if (cap < (uint32_t)nauc) throw ReadFail{ASD_EINVAL, "atoms[] holds fewer entries than the unit cell"};
        std::vector<double> base_mu((size_t)nms, -1.0);
        for (long long i = 0; i < nauc; i++) {
            asd_ucf_atom a{};
            long long sl = -1;
            in >> sl >> a.xred[0] >> a.xred[1] >> a.xred[2];
            if (mesh_points) in >> a.mesh_point[0] >> a.mesh_point[1] >> a.mesh_point[2];
            in >> a.mu >> a.damping >> a.gamma;
            std::string el;
            in >> el >> a.init_spin[0] >> a.init_spin[1] >> a.init_spin[2] >> a.k1u >> a.k1u_dir[0] >> a.k1u_dir[1] >>
                a.k1u_dir[2];
            if (!in) throw ReadFail{ASD_EINVAL, "Unit cell file ended early or is not of the correct format (atom " +
                                                    std::to_string(i) + ")"};
            // a species number must index the nms sublattices (the reference's check, s > nms,
            // src/unitcell.h:124, also lets s == nms through)
            if (sl < 0 || sl >= nms)
                throw ReadFail{ASD_EINVAL, "an atom in the unit cell has a species number not below the number of "
                                           "sublattices"};
            a.sublattice = (uint32_t)sl;
            std::snprintf(a.element, sizeof a.element, "%s", el.c_str());
            if (a.mu < 1e-5) throw ReadFail{ASD_EINVAL, "Magnetic moment is less than 1e-5 (so, very small)."};
            if (a.mu > 1e5) throw ReadFail{ASD_EINVAL, "Magnetic moment is greater than 1e5 (so, really huge)."};
            if (a.gamma < 1e-5) throw ReadFail{ASD_EINVAL, "Gyromagnetic is less than 1e-5 (so, really small)."};
            if (a.gamma > 1e5) throw ReadFail{ASD_EINVAL, "Gyromagnetic is greater than 1e5 (so, really huge)."};
            const double m = std::sqrt(a.k1u_dir[0] * a.k1u_dir[0] + a.k1u_dir[1] * a.k1u_dir[1] +
                                       a.k1u_dir[2] * a.k1u_dir[2]);
            if (std::fabs(m - 1) > 1e-6)   // src/unitcell.h:137
                throw ReadFail{ASD_EINVAL, "The input direction for the uniaxial anisotropy constant must have a "
                                           "modulus of 1 (atom " + std::to_string(i) + ")"};
            if (base_mu[a.sublattice] < 0) base_mu[a.sublattice] = a.mu;
            atoms[i] = a;
        }
        for (long long i = 0; i < nauc; i++)   // unitCellMembers::CheckSpecies (src/unitcell.h:187-218)
            if (std::fabs(atoms[i].mu - base_mu[atoms[i].sublattice]) > 1e-12)
                throw ReadFail{ASD_EINVAL, "A magnetic moment was associated with an atom in the unit cell whose "
                                           "magnetic moment is not consistent with others in that species."};
    } catch (const ReadFail& f) {
        put_err(err, err_len, f.msg);
        return f.code;
    }
    return ASD_OK;
}

int asd_read_exch(const char* path, uint32_t nms, uint32_t* nbonds, uint32_t* bond_s1, uint32_t* bond_s2,
                  int32_t* bond_vec, double* bond_J, uint32_t cap, char* err, size_t err_len) {
    try {
        if (!path || !nbonds || nms == 0) throw ReadFail{ASD_EINVAL, "path, nbonds and nms > 0 are required"};
        std::ifstream in(path);
        if (!in) throw ReadFail{ASD_EINVAL, std::string("Could not open exchange file ") + path};
        std::stringstream ss;
        ss << in.rdbuf();
        Cfg cfg(ss.str());
        cfg.parse();
        uint32_t nb = 0;
        const bool fill = bond_s1 && bond_s2 && bond_vec && bond_J;
        for (uint32_t s1 = 0; s1 < nms; s1++) {
            for (uint32_t s2 = 0; s2 < nms; s2++) {
                const std::string g = "exchange_" + std::to_string(s1) + "_" + std::to_string(s2);
                if (!cfg.has_group(g)) continue;   // an absent pair has no interactions
                std::string t;
                if (!cfg.scalar(g + ".Num_Interactions", &t))
                    throw ReadFail{ASD_EINVAL, "Could not read the number of interactions between species " +
                                                   std::to_string(s1) + " and " + std::to_string(s2)};
                const double nint_d = to_double(t, g + ".Num_Interactions");
                if (nint_d < 0 || nint_d != std::floor(nint_d)) throw ReadFail{ASD_EINVAL, g + ".Num_Interactions"};
                const uint32_t nint = (uint32_t)nint_d;
                std::string units = "joules";   // the reference warns and defaults to joules
                cfg.scalar(g + ".units", &units);
                const double uf = unit_factor(units);
                for (uint32_t i = 0; i < nint; i++) {
                    std::vector<std::string> v;
                    const std::string uc = g + ".UnitCell" + std::to_string(i + 1);
                    if (!cfg.array(uc, &v) || v.size() < 3)
                        throw ReadFail{ASD_EINVAL, "Could not read vector for interaction number " + std::to_string(i + 1) +
                                                       " (between " + std::to_string(s1) + " and " + std::to_string(s2) + ")"};
                    double Jm[9];
                    for (int r = 0; r < 3; r++) {
                        std::vector<std::string> row;
                        const std::string jr = g + ".J" + std::to_string(i + 1) + "_" + std::to_string(r + 1);
                        if (!cfg.array(jr, &row) || row.size() < 3)
                            throw ReadFail{ASD_EINVAL, "Could not read exchange interaction " + jr};
                        for (int c = 0; c < 3; c++) Jm[3 * r + c] = to_double(row[c], jr) * uf;
                    }
                    if (fill) {
                        if (nb >= cap) throw ReadFail{ASD_EINVAL, "bond arrays hold fewer entries than the file"};
                        bond_s1[nb] = s1;
                        bond_s2[nb] = s2;
                        for (int c = 0; c < 3; c++) bond_vec[3 * nb + c] = round_offset(to_double(v[c], uc));
                        for (int q = 0; q < 9; q++) bond_J[9 * (size_t)nb + q] = Jm[q];
                    }
                    nb++;
                }
            }
        }
        *nbonds = nb;
    } catch (const ReadFail& f) {
        put_err(err, err_len, f.msg);
        return f.code;
    }
    return ASD_OK;
}

int asd_read_csr_exch(const char* path, uint32_t nspins, uint32_t* nnz_out, uint32_t* xadj, uint32_t* adjncy,
                      double* val9, uint32_t cap, char* err, size_t err_len) {
    try {
        if (!path || !nnz_out) throw ReadFail{ASD_EINVAL, "path and nnz are required"};
        std::ifstream in(path);
        if (!in) throw ReadFail{ASD_EINVAL, "You requested to read in a CSR exchange matrix but it does not exist"};
        unsigned long long lns = 0, adjsize = 0;
        in >> lns >> adjsize;
        if (!in || lns != nspins)
            throw ReadFail{ASD_EINVAL, "The number of spins (first line) in the CSR input file is not consistent with "
                                       "the system size. (First check failed)"};
        if (adjsize < 1) throw ReadFail{ASD_EINVAL, "The size of adjncy (neighbour list) is zero. (Second check failed)"};
        if (adjsize > 0xFFFFFFFFull) throw ReadFail{ASD_EINVAL, "adjncy too large"};
        *nnz_out = (uint32_t)adjsize;
        if (!xadj) return ASD_OK;
        if (!adjncy || !val9 || cap < adjsize) throw ReadFail{ASD_EINVAL, "output arrays hold fewer entries than the file"};
        for (uint32_t i = 0; i <= nspins; i++) in >> xadj[i];
        if (!in) throw ReadFail{ASD_EINVAL, "CSR file ended inside xadj"};
        for (uint32_t i = 0; i < nspins; i++)
            if (xadj[i] > xadj[i + 1] || xadj[i + 1] > adjsize)
                throw ReadFail{ASD_EINVAL, "There is an error in the xadj lookup. (Third check failed)"};
        std::memset(val9, 0, sizeof(double) * 9 * (size_t)adjsize);
        for (uint32_t i = 0; i < nspins; i++)
            for (uint32_t j = xadj[i]; j < xadj[i + 1]; j++) {
                in >> adjncy[j] >> val9[9 * (size_t)j] >> val9[9 * (size_t)j + 4] >> val9[9 * (size_t)j + 8];
                if (!in) throw ReadFail{ASD_EINVAL, "CSR file ended inside the entries"};
                if (adjncy[j] >= nspins) throw ReadFail{ASD_EINVAL, "CSR column index out of range"};
            }
    } catch (const ReadFail& f) {
        put_err(err, err_len, f.msg);
        return f.code;
    }
    return ASD_OK;
}

int asd_write_csr_exch(const char* path, uint32_t nspins, const uint32_t* xadj, const uint32_t* adjncy,
                       const double* val9) {
    if (!path || !xadj || !adjncy || !val9) return ASD_EINVAL;
    FILE* f = std::fopen(path, "w");
    if (!f) return ASD_EINVAL;
    std::fprintf(f, "%u\n%u\n", nspins, xadj[nspins]);
    for (uint32_t i = 0; i < nspins; i++) std::fprintf(f, "%u\t", xadj[i]);
    std::fprintf(f, "%u\n", xadj[nspins]);
    for (uint32_t i = 0; i < nspins; i++)
        for (uint32_t j = xadj[i]; j < xadj[i + 1]; j++)
            std::fprintf(f, "%u\t%.17g\t%.17g\t%.17g\t", adjncy[j], val9[9 * (size_t)j], val9[9 * (size_t)j + 4],
                         val9[9 * (size_t)j + 8]);
    const bool ok = std::fclose(f) == 0;
    return ok ? ASD_OK : ASD_EINVAL;
}

}  // extern "C"
