// Native input layer: basis files, molecule inputs and the shell layout that
// hfgpu_init consumes (include/hfgpu_ingest.h).  Host code only.
//
// Restates, in the reference's conventions:
//   read_basfile.f90:1-96     basis-file grammar: header "ELEMENTS n dmat",
//                             per element a shell count, a label, per shell
//                             "TYPE nprim [scale]" and nprim rows "zeta c"
//                             (or "zeta c_s c_p" for L), a "****" line; with
//                             dmat = 1 a density section follows, one
//                             nbf x nbf block per element written row by row
//   read_basfile.f90:100-179  normalize: primitive norms folded into the
//                             coefficients, then the contracted shell scaled
//                             to unit norm (d: the x^2 component's norm)
//   read_infile.f90:12-61     molecule input: natom, title, keyword lines,
//                             then "label x y z" in Angstrom.  The keyword
//                             lines are taken in any order up to the first
//                             atom line, so the older headers the reference
//                             ships (HUCKEL, no DIRECTSCF, CRLF) also load
//   read_infile.f90:122-149   element label -> nuclear charge (H..Kr)
//   spread_basis.f90:66-182   shells atom-major in basis-file order, AO
//                             offsets in the same walk, djkl = c_p / c_s for
//                             L shells, mixed P + D + L rejected
//   nuclear_repulsion.f90     sum_{i<j} Z_i Z_j / r_ij
//   direct_hartreefock.f90:50-59  block-diagonal atomic density guess
//
// Fortran list-directed reads consume whole records: a read takes its items
// from as many lines as it needs (blank lines are skipped) and drops the rest
// of the last line.  Reader::items() does the same.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/hfgpu_ingest.h"

namespace hfgpu {
void set_last_error(const std::string& msg);  // hfgpu.cu
}

namespace {

const int MAXPRIM = 10;              // molprops.f90:19
const double BOHR = 1.889725989;     // read_infile.f90:6
const double PI = 3.141592653589793238462643383279502884197;

const char* const ELEMENTS[36] = {"h",  "he", "li", "be", "b",  "c",  "n",  "o",  "f",  "ne", "na", "mg",
                                  "al", "si", "p",  "s",  "cl", "ar", "k",  "ca", "sc", "ti", "v",  "cr",
                                  "mn", "fe", "co", "ni", "cu", "zn", "ga", "ge", "as", "se", "br", "kr"};

std::string lower(std::string s) {
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

int nfunc_of(int t) { return t == HFGPU_SHELL_S ? 1 : t == HFGPU_SHELL_P ? 3 : t == HFGPU_SHELL_D ? 5 : 4; }

int atomic_number(const std::string& label) {
    const std::string l = lower(label);
    for (int i = 0; i < 36; ++i)
        if (l == ELEMENTS[i]) return i + 1;
    throw std::runtime_error("element not recognized: '" + label + "'");
}

// Record-oriented token reader (Fortran list-directed input).
class Reader {
  public:
    explicit Reader(const std::string& path) : path_(path) {
        std::ifstream in(path);
        if (!in) throw std::runtime_error("cannot open " + path);
        std::string ln;
        while (std::getline(in, ln)) {
            if (!ln.empty() && ln.back() == '\r') ln.pop_back();  // CRLF files
            lines_.push_back(ln);
        }
    }
    // The next n whitespace-separated items, starting on a fresh line.
    std::vector<std::string> items(size_t n) {
        std::vector<std::string> out;
        while (out.size() < n) {
            if (pos_ >= lines_.size())
                throw std::runtime_error(path_ + ": unexpected end of file");
            std::istringstream ss(lines_[pos_++]);
            std::string t;
            while (out.size() < n && ss >> t) out.push_back(t);
        }
        return out;
    }
    // The next non-blank line split into tokens (all of them).
    std::vector<std::string> line() {
        while (pos_ < lines_.size()) {
            std::istringstream ss(lines_[pos_++]);
            std::vector<std::string> t;
            std::string s;
            while (ss >> s) t.push_back(s);
            if (!t.empty()) return t;
        }
        throw std::runtime_error(path_ + ": unexpected end of file");
    }
    std::vector<std::string> peek() {
        size_t keep = pos_;
        std::vector<std::string> t = line();
        pos_ = keep;
        return t;
    }
    const std::string& path() const { return path_; }

  private:
    std::string path_;
    std::vector<std::string> lines_;
    size_t pos_ = 0;
};

double to_d(const std::string& s, const std::string& where) {
    std::string t = s;
    for (char& c : t)
        if (c == 'd' || c == 'D') c = 'e';  // Fortran double exponent
    char* end = nullptr;
    const double v = std::strtod(t.c_str(), &end);
    if (end == t.c_str() || *end != '\0') throw std::runtime_error(where + ": not a number: '" + s + "'");
    return v;
}

int to_i(const std::string& s, const std::string& where) {
    char* end = nullptr;
    const long v = std::strtol(s.c_str(), &end, 10);
    if (end == s.c_str() || *end != '\0') throw std::runtime_error(where + ": not an integer: '" + s + "'");
    return (int)v;
}

// read_basfile.f90:100-179.  l = 0, 1, 2; coefficients updated in place.
void normalize(int n, const double* zeta, int l, double* c) {
    for (int k = 0; k < n; ++k) {
        const double a = zeta[k];
        if (l == 0) c[k] *= std::pow(2.0 * a / PI, 0.75);
        else if (l == 1) c[k] *= std::pow(2.0 / PI, 0.75) * 2.0 * std::pow(a, 1.25);
        else c[k] *= std::pow(2.0 / PI, 0.75) * 4.0 * std::pow(a, 1.75) / std::sqrt(3.0);
    }
    const double pi32 = std::sqrt(PI * PI * PI);
    double nfac = 0.0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const double p = zeta[i] + zeta[j];
            double o;
            if (l == 0) o = pi32 / std::sqrt(p * p * p);
            else if (l == 1) o = pi32 / (2.0 * p * p * std::sqrt(p));
            else o = pi32 * 3.0 / (4.0 * p * p * p * std::sqrt(p));
            nfac += o * c[i] * c[j];
        }
    const double s = 1.0 / std::sqrt(nfac);
    for (int k = 0; k < n; ++k) c[k] *= s;
}

struct ElShell {
    int typ;
    int nz;
    double zeta[MAXPRIM];
    double cs[MAXPRIM];  // s (or the only) coefficients, normalised
    double cp[MAXPRIM];  // L shells: p coefficients, normalised
};

struct Element {
    std::string label;
    std::vector<ElShell> shells;
    std::vector<double> dmat;  // nbf x nbf, row-major as written
    int nbf = 0;
};

struct BasFile {
    std::vector<Element> el;
    bool dmat = false;
    const Element* find(const std::string& label) const {
        const std::string l = lower(label);
        for (const Element& e : el)
            if (e.label == l) return &e;
        return nullptr;
    }
};

BasFile read_basfile(const std::string& path) {
    Reader r(path);
    BasFile b;
    std::vector<std::string> h = r.items(3);
    const int nel = to_i(h[1], path);
    b.dmat = to_i(h[2], path) != 0;
    for (int i = 0; i < nel; ++i) {
        Element e;
        const int nsh = to_i(r.items(1)[0], path);
        e.label = lower(r.items(1)[0]);
        for (int j = 0; j < nsh; ++j) {
            std::vector<std::string> t = r.items(2);
            const std::string ty = lower(t[0]);
            ElShell s{};
            s.nz = to_i(t[1], path);
            if (s.nz < 1 || s.nz > MAXPRIM)
                throw std::runtime_error(path + ": element " + e.label + ": primitive count out of range");
            int l;
            if (ty == "s") { s.typ = HFGPU_SHELL_S; l = 0; }
            else if (ty == "p") { s.typ = HFGPU_SHELL_P; l = 1; }
            else if (ty == "d") { s.typ = HFGPU_SHELL_D; l = 2; }
            else if (ty == "l") { s.typ = HFGPU_SHELL_L; l = 12; }
            else throw std::runtime_error(path + ": unknown shell type '" + t[0] + "'");
            for (int k = 0; k < s.nz; ++k) {
                std::vector<std::string> v = r.items(l == 12 ? 3 : 2);
                s.zeta[k] = to_d(v[0], path);
                s.cs[k] = to_d(v[1], path);
                s.cp[k] = l == 12 ? to_d(v[2], path) : 0.0;
            }
            if (l == 12) {
                normalize(s.nz, s.zeta, 0, s.cs);
                normalize(s.nz, s.zeta, 1, s.cp);
            } else {
                normalize(s.nz, s.zeta, l, s.cs);
            }
            e.nbf += nfunc_of(s.typ);
            e.shells.push_back(s);
        }
        if (r.items(1)[0].rfind("****", 0) != 0)
            throw std::runtime_error(path + ": element " + e.label + " not closed by ****");
        b.el.push_back(e);
    }
    if (b.dmat) {
        r.items(1);  // "DENSITY MATRICES"
        for (Element& e : b.el) {
            r.items(1);  // element label
            const int n = e.nbf;
            e.dmat.assign((size_t)n * n, 0.0);
            // each row ii is written in records of at most 7 values
            for (int ii = 0; ii < n; ++ii)
                for (int kk = 0; kk < n; kk += 7) {
                    const int m = n - kk < 7 ? n - kk : 7;
                    std::vector<std::string> v = r.items(m);
                    for (int q = 0; q < m; ++q) e.dmat[(size_t)ii * n + kk + q] = to_d(v[q], path);
                }
            if (r.items(1)[0].rfind("****", 0) != 0)
                throw std::runtime_error(path + ": density block of " + e.label + " not closed by ****");
        }
    }
    return b;
}

bool is_atom_line(const std::vector<std::string>& t) {
    if (t.size() < 4 || !std::isalpha((unsigned char)t[0][0])) return false;
    for (int k = 1; k < 4; ++k) {
        try {
            to_d(t[k], "");
        } catch (const std::exception&) {
            return false;
        }
    }
    return true;
}

bool yes(const std::vector<std::string>& t, size_t k) {
    return t.size() > k && !t[k].empty() && std::tolower((unsigned char)t[k][0]) == 'y';
}

}  // namespace

struct hfgpu_system {
    hfgpu_system_info info{};
    std::vector<int> z, nbfat;
    std::vector<double> xyz;  // bohr, natom x 3
    std::vector<int> shtyp, nzet, atsh, aosh;
    std::vector<double> xsh, zeta, djk, djkl;
    std::vector<std::vector<double>> dmat;  // per atom, row-major nbf x nbf
};

namespace {

void read_infile(const std::string& path, hfgpu_system& s, std::vector<std::string>& labels,
                 std::vector<double>& ang) {
    Reader r(path);
    const int natom = to_i(r.items(1)[0], path);
    if (natom < 1) throw std::runtime_error(path + ": no atoms");
    r.line();  // title
    hfgpu_system_info& o = s.info;
    o.directscf = 1;
    while (!is_atom_line(r.peek())) {
        std::vector<std::string> t = r.line();
        const std::string key = lower(t[0]);
        if (key == "usedensitysupguess") o.densup = yes(t, 1);
        else if (key == "directscf") o.directscf = yes(t, 1);
        else if (key == "levelshift") {
            o.levshft = yes(t, 1);
            o.lshft = t.size() > 2 ? to_d(t[2], path) : 0.0;
        } else if (key == "uhf") {
            o.uhf = yes(t, 1);
            o.sz = t.size() > 2 ? to_i(t[2], path) : 0;
        } else if (key == "mp2") o.mp2 = yes(t, 1);
        else if (key == "ccsd") o.ccsd = yes(t, 1);
        else if (key == "huckel") o.huckel = yes(t, 1);
        else if (key == "print") o.prtlevl = t.size() > 1 ? to_i(t[1], path) : 0;
        else if (key == "ncore") o.ncore = t.size() > 1 ? to_i(t[1], path) : 0;
        else throw std::runtime_error(path + ": unknown header line starting '" + t[0] + "'");
    }
    for (int i = 0; i < natom; ++i) {
        std::vector<std::string> t = r.line();
        if (!is_atom_line(t)) throw std::runtime_error(path + ": bad atom line starting '" + t[0] + "'");
        labels.push_back(t[0]);
        for (int k = 1; k < 4; ++k) ang.push_back(to_d(t[k], path));
    }
}

// spread_basis.f90:66-182 plus the per-atom data the builders and the SCF
// read (charges, coordinates, nuclear repulsion, density blocks).
void spread(const BasFile& b, const std::vector<std::string>& labels, const std::vector<double>& ang,
            hfgpu_system& s) {
    const int natom = (int)labels.size();
    s.info.natom = natom;
    s.info.maxprim = MAXPRIM;
    s.info.has_density = b.dmat ? 1 : 0;
    int iao = 0, nelec = 0;
    bool hasp = false, hasd = false, hasl = false;
    for (int ia = 0; ia < natom; ++ia) {
        const int zn = atomic_number(labels[ia]);
        const Element* e = b.find(labels[ia]);
        if (!e) throw std::runtime_error("element " + labels[ia] + " not in basis");
        nelec += zn;
        s.z.push_back(zn);
        s.nbfat.push_back(e->nbf);
        double x[3];
        for (int k = 0; k < 3; ++k) {
            x[k] = ang[3 * ia + k] * BOHR;
            s.xyz.push_back(x[k]);
        }
        for (const ElShell& sh : e->shells) {
            s.shtyp.push_back(sh.typ);
            s.nzet.push_back(sh.nz);
            s.atsh.push_back(ia);
            s.aosh.push_back(iao);
            for (int k = 0; k < 3; ++k) s.xsh.push_back(x[k]);
            for (int k = 0; k < MAXPRIM; ++k) {
                const bool on = k < sh.nz;
                s.zeta.push_back(on ? sh.zeta[k] : 0.0);
                s.djk.push_back(on ? sh.cs[k] : 0.0);
                s.djkl.push_back(on && sh.typ == HFGPU_SHELL_L ? sh.cp[k] / sh.cs[k] : 0.0);
            }
            hasp |= sh.typ == HFGPU_SHELL_P;
            hasd |= sh.typ == HFGPU_SHELL_D;
            hasl |= sh.typ == HFGPU_SHELL_L;
            iao += nfunc_of(sh.typ);
        }
        s.dmat.push_back(e->dmat);
    }
    if (hasp && hasd && hasl) throw std::runtime_error("Mixed P, D and L shells not supported");
    s.info.nsh = (int)s.shtyp.size();
    s.info.nb = iao;
    s.info.nelec = nelec;
    s.info.nocc = nelec / 2;
    double en = 0.0;
    for (int i = 0; i < natom; ++i)
        for (int j = i + 1; j < natom; ++j) {
            double r2 = 0.0;
            for (int k = 0; k < 3; ++k) {
                const double d = s.xyz[3 * i + k] - s.xyz[3 * j + k];
                r2 += d * d;
            }
            en += (double)s.z[i] * s.z[j] / std::sqrt(r2);
        }
    s.info.enuc = en;
}

int fail(const std::string& what, const std::exception& e) {
    hfgpu::set_last_error(what + ": " + e.what());
    return 1;
}

}  // namespace

extern "C" {

int hfgpu_system_from_files(const char* basfile, const char* infile, hfgpu_system** out) {
    if (!basfile || !infile || !out) {
        hfgpu::set_last_error("hfgpu_system_from_files: bad arguments");
        return 1;
    }
    *out = nullptr;
    try {
        BasFile b = read_basfile(basfile);
        hfgpu_system* s = new hfgpu_system();
        std::vector<std::string> labels;
        std::vector<double> ang;
        try {
            read_infile(infile, *s, labels, ang);
            spread(b, labels, ang, *s);
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
        return 0;
    } catch (const std::exception& e) {
        return fail("hfgpu_system_from_files", e);
    }
}

int hfgpu_system_from_atoms(const char* basfile, int natom, const char* const* labels, const double* coords_ang,
                            hfgpu_system** out) {
    if (!basfile || natom < 1 || !labels || !coords_ang || !out) {
        hfgpu::set_last_error("hfgpu_system_from_atoms: bad arguments");
        return 1;
    }
    *out = nullptr;
    try {
        BasFile b = read_basfile(basfile);
        std::vector<std::string> lab;
        for (int i = 0; i < natom; ++i) {
            if (!labels[i]) throw std::runtime_error("null label");
            lab.push_back(labels[i]);
        }
        std::vector<double> ang(coords_ang, coords_ang + 3 * (size_t)natom);
        hfgpu_system* s = new hfgpu_system();
        s->info.directscf = 1;
        try {
            spread(b, lab, ang, *s);
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
        return 0;
    } catch (const std::exception& e) {
        return fail("hfgpu_system_from_atoms", e);
    }
}

int hfgpu_system_get_info(const hfgpu_system* s, hfgpu_system_info* info) {
    if (!s || !info) {
        hfgpu::set_last_error("hfgpu_system_get_info: bad arguments");
        return 1;
    }
    *info = s->info;
    return 0;
}

int hfgpu_system_basis(const hfgpu_system* s, hfgpu_basis* v) {
    if (!s || !v) {
        hfgpu::set_last_error("hfgpu_system_basis: bad arguments");
        return 1;
    }
    v->nsh = s->info.nsh;
    v->nb = s->info.nb;
    v->maxprim = MAXPRIM;
    v->shtyp = s->shtyp.data();
    v->nzet = s->nzet.data();
    v->atsh = s->atsh.data();
    v->aosh = s->aosh.data();
    v->xsh = s->xsh.data();
    v->zeta = s->zeta.data();
    v->djk = s->djk.data();
    v->djkl = s->djkl.data();
    return 0;
}

int hfgpu_system_atoms(const hfgpu_system* s, int* charges, double* coords_bohr) {
    if (!s) {
        hfgpu::set_last_error("hfgpu_system_atoms: bad arguments");
        return 1;
    }
    if (charges) std::memcpy(charges, s->z.data(), s->z.size() * sizeof(int));
    if (coords_bohr) std::memcpy(coords_bohr, s->xyz.data(), s->xyz.size() * sizeof(double));
    return 0;
}

int hfgpu_system_atom_nbf(const hfgpu_system* s, int* nbf) {
    if (!s || !nbf) {
        hfgpu::set_last_error("hfgpu_system_atom_nbf: bad arguments");
        return 1;
    }
    std::memcpy(nbf, s->nbfat.data(), s->nbfat.size() * sizeof(int));
    return 0;
}

int hfgpu_system_density_guess(const hfgpu_system* s, double* p) {
    if (!s || !p) {
        hfgpu::set_last_error("hfgpu_system_density_guess: bad arguments");
        return 1;
    }
    if (!s->info.has_density) {
        hfgpu::set_last_error("hfgpu_system_density_guess: basis file has no density matrices");
        return 1;
    }
    const size_t nb = (size_t)s->info.nb;
    std::memset(p, 0, nb * nb * sizeof(double));
    size_t k = 0;
    for (size_t a = 0; a < s->nbfat.size(); ++a) {
        const size_t n = (size_t)s->nbfat[a];
        const std::vector<double>& d = s->dmat[a];
        for (size_t i = 0; i < n; ++i)
            for (size_t j = 0; j < n; ++j) p[(k + j) * nb + (k + i)] = d[i * n + j];  // P(k+i, k+j)
        k += n;
    }
    return 0;
}

void hfgpu_system_free(hfgpu_system* s) { delete s; }

}  // extern "C"
