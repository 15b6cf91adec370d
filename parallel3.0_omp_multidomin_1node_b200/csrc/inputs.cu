// Reference case files read into the library's problem description: the
// datacard BEM_DATACARD.DAT (GMRES solver card with the optional multi-domain
// tail), input/<title>.model and input/<title>.bd in text form or in the
// DBEMBIN binary form (<file>.bin), and the batch boundary files of the
// card's batch modes, which become load cases.  Host code only.
//
//   datacard          DBEM1/DBEM.cpp:637-791
//   multi-domain tail DBEM1/multidomain.cpp:1305-1362, ids and defaults
//                     DBEM1/multidomain.cpp:500-523, 1363-1477
//   .model / .bd text DBEM1/DBEM.cpp:826-1085, 295-343
//   DBEMBIN           DBEM1/DBEM.cpp:89-293
#include "../../include/tdbem.h"
#include "host_error.h"

#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

struct tdbem_case {
    std::string title;
    std::vector<double> points;
    std::vector<int64_t> elements;
    std::vector<int32_t> bcid;
    std::vector<double> materials;    // [domains][3] E, nu, rho
    std::vector<int64_t> interfaces;  // [I][5] 0-based
    double card_E = 0, card_nu = 0, card_rho = 0, beta = 0, gap = 0, tol = 0;
    int32_t n_steps = 0, restart = 0, max_leaf = 0, threads = 0, n_domains = 1, n_loads = 1;
    std::vector<double> known;        // [n_loads][n_steps + 1][E][3]
};

namespace {

// Whitespace-separated tokens of a text file, read like fscanf's %s / %d / %lf.
struct Tokens {
    std::vector<std::string> t;
    size_t pos = 0;
    bool load(const std::string& path)
    {
        FILE* f = std::fopen(path.c_str(), "rb");
        if (!f) return false;
        std::string s;
        char buf[1 << 16];
        size_t n;
        while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) s.append(buf, n);
        std::fclose(f);
        size_t i = 0;
        while (i < s.size()) {
            while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
            size_t j = i;
            while (j < s.size() && !std::isspace((unsigned char)s[j])) ++j;
            if (j > i) t.emplace_back(s.substr(i, j - i));
            i = j;
        }
        return true;
    }
    bool more() const { return pos < t.size(); }
    bool str(std::string& v)
    {
        if (!more()) return false;
        v = t[pos++];
        return true;
    }
    bool i64(long long& v)
    {
        if (!more()) return false;
        errno = 0;
        char* e = nullptr;
        v = std::strtoll(t[pos].c_str(), &e, 10);
        if (e == t[pos].c_str() || *e || errno) return false;
        ++pos;
        return true;
    }
    bool f64(double& v)
    {
        if (!more()) return false;
        char* e = nullptr;
        v = std::strtod(t[pos].c_str(), &e);
        if (e == t[pos].c_str() || *e) return false;
        ++pos;
        return true;
    }
};

tdbem_status bad(const std::string& m)
{
    tdbem::set_last_error(m);
    return TDBEM_INVALID_INPUT;
}

bool file_exists(const std::string& p)
{
    FILE* f = std::fopen(p.c_str(), "rb");
    if (!f) return false;
    std::fclose(f);
    return true;
}

constexpr char kMagic[8] = {'D', 'B', 'E', 'M', 'B', 'I', 'N', '\0'};

bool binary_header(FILE* f, uint32_t kind)
{
    char magic[8];
    uint32_t h[4];
    if (std::fread(magic, 1, 8, f) != 8 || std::fread(h, sizeof(uint32_t), 4, f) != 4) return false;
    return std::memcmp(magic, kMagic, 8) == 0 && h[0] == 1 && h[1] == kind && h[2] == 0x01020304u;
}

tdbem_status read_model_text(const std::string& path, tdbem_case& c)
{
    Tokens t;
    if (!t.load(path)) return bad("cannot open model file " + path);
    long long np = 0, ne = 0;
    if (!t.i64(np) || np <= 0) return bad("invalid point count in " + path);
    c.points.resize((size_t)np * 3);
    for (auto& v : c.points)
        if (!t.f64(v)) return bad("invalid point data in " + path);
    if (!t.i64(ne) || ne <= 0) return bad("invalid element count in " + path);
    c.elements.resize((size_t)ne * 8);
    for (auto& v : c.elements) {
        long long id;
        if (!t.i64(id)) return bad("invalid element data in " + path);
        v = id - 1;  // 1-based point ids in the text form
    }
    return TDBEM_OK;
}

tdbem_status read_model_binary(const std::string& path, tdbem_case& c)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return bad("cannot open binary model file " + path);
    tdbem_status st = TDBEM_OK;
    int64_t n = 0;
    if (!binary_header(f, 1)) {
        st = bad("binary header mismatch in " + path);
    } else if (std::fread(&n, 8, 1, f) != 1 || n <= 0) {
        st = bad("invalid point count in " + path);
    } else {
        c.points.resize((size_t)n * 3);
        if (std::fread(c.points.data(), sizeof(double), c.points.size(), f) != c.points.size() ||
            std::fread(&n, 8, 1, f) != 1 || n <= 0) {
            st = bad("invalid point or element section in " + path);
        } else {
            c.elements.resize((size_t)n * 8);  // 0-based point ids in the binary form
            if (std::fread(c.elements.data(), sizeof(int64_t), c.elements.size(), f) != c.elements.size())
                st = bad("invalid element data in " + path);
        }
    }
    std::fclose(f);
    return st;
}

// One boundary file: BCIDs, then (n_steps + 1) x E x 3 prescribed values.
// With `expect`, the BCIDs must equal it.
tdbem_status read_bd(const std::string& path, bool binary, int64_t E, int32_t n_steps, std::vector<int32_t>& bcid,
                     const std::vector<int32_t>* expect, double* out)
{
    const size_t nv = (size_t)(n_steps + 1) * E * 3;
    std::vector<int32_t> ids((size_t)E);
    if (binary) {
        FILE* f = std::fopen(path.c_str(), "rb");
        if (!f) return bad("cannot open binary boundary file " + path);
        int64_t fe = 0, fn = 0;
        bool ok = binary_header(f, 2) && std::fread(&fe, 8, 1, f) == 1 && std::fread(&fn, 8, 1, f) == 1 && fe == E &&
                  fn == n_steps && std::fread(ids.data(), sizeof(int32_t), ids.size(), f) == ids.size() &&
                  std::fread(out, sizeof(double), nv, f) == nv;
        std::fclose(f);
        if (!ok) return bad("invalid or mismatched binary boundary file " + path);
    } else {
        Tokens t;
        if (!t.load(path)) return bad("cannot open boundary file " + path);
        for (auto& b : ids) {
            long long v;
            if (!t.i64(v)) return bad("invalid boundary type section in " + path);
            b = (int32_t)v;
        }
        for (size_t i = 0; i < nv; ++i)
            if (!t.f64(out[i])) return bad("invalid boundary value section in " + path);
    }
    if (expect && ids != *expect) return bad("boundary types in " + path + " differ from the first load case");
    bcid = ids;
    return TDBEM_OK;
}

int normalize_domain(long long id, int count, bool zero_based)
{
    if (zero_based && id >= 0 && id < count) return (int)id;
    if (id >= 1 && id <= count) return (int)id - 1;
    return -1;
}

long long normalize_element(long long id, long long n, bool zero_based)
{
    if (zero_based) return (id >= 0 && id < n) ? id : -1;
    return (id >= 1 && id <= n) ? id - 1 : -1;
}

}  // namespace

extern "C" {

tdbem_status tdbem_case_read(const char* directory, tdbem_case** out)
{
    tdbem::set_last_error("");
    if (!directory || !out) return bad("null argument");
    *out = nullptr;
    const std::string dir = std::string(directory) + "/";
    Tokens t;
    if (!t.load(dir + "BEM_DATACARD.DAT")) return bad("cannot open " + dir + "BEM_DATACARD.DAT");
    tdbem_case c;
    long long threads, flag_dyna, nstep, solver, iterations, premax, mode_a, mode_b;
    double amplitude;
    if (!t.str(c.title) || !t.i64(threads) || !t.i64(flag_dyna) || !t.f64(c.beta) || !t.i64(nstep) ||
        !t.f64(c.gap) || !t.f64(c.card_E) || !t.f64(c.card_nu) || !t.f64(c.card_rho) || !t.f64(amplitude) ||
        !t.i64(solver))
        return bad("datacard header incomplete");
    if (solver != 2) return bad("only the GMRES solver card (solvers = 2) drives the multi-domain march");
    if (!t.i64(iterations) || !t.f64(c.tol) || !t.i64(premax)) return bad("GMRES card incomplete");
    c.threads = (int32_t)threads;
    c.n_steps = (int32_t)nstep;
    c.restart = (int32_t)iterations;
    c.max_leaf = (int32_t)premax;
    // input mode and batch boundary mode, with the reference's tolerance for
    // cards that give only one of them or the batch count in their place
    int input_mode = 0, batch_mode = 0;
    long long pre_count = -1;
    if (t.i64(mode_a)) {
        if (mode_a < 0 || mode_a > 2) {
            batch_mode = (int)mode_a;
        } else {
            input_mode = (int)mode_a;
            if (t.i64(mode_b)) {
                if (mode_b < 0 || mode_b > 2) {
                    pre_count = mode_b;
                    batch_mode = input_mode;
                    input_mode = 0;
                } else {
                    batch_mode = (int)mode_b;
                }
            }
        }
    }
    std::vector<std::string> batch_files;
    if (batch_mode == 1 || batch_mode == 2) {
        long long count = pre_count;
        if (count <= 0 && !t.i64(count)) return bad("batch boundary count missing");
        if (batch_mode == 1) {
            for (long long i = 0; i < count; ++i) {
                std::string s;
                if (!t.str(s)) return bad("batch boundary file list incomplete");
                batch_files.push_back(s);
            }
        } else {
            std::string bdir, prefix, ext;
            long long first, last;
            if (!t.str(bdir) || !t.str(prefix) || !t.i64(first) || !t.i64(last) || !t.str(ext))
                return bad("batch boundary directory card incomplete");
            if (count <= 0 || last < first) return bad("invalid batch boundary directory card");
            for (long long i = 0; i < count; ++i)
                batch_files.push_back(bdir + prefix + std::to_string(first + i) + ext);
        }
    }
    // optional multi-domain tail
    long long ndom = 1;
    std::vector<long long> mid;
    std::vector<double> mval;
    std::vector<long long> itf_raw;
    bool tail = t.i64(ndom);
    if (tail) {
        if (ndom <= 0) return bad("invalid DomainCount " + std::to_string(ndom));
        for (long long i = 0; i < ndom; ++i) {
            long long id;
            double e, v, r;
            if (!t.i64(id) || !t.f64(e) || !t.f64(v) || !t.f64(r))
                return bad("invalid material line for domain " + std::to_string(i));
            mid.push_back(id);
            mval.insert(mval.end(), {e, v, r});
        }
        long long nitf;
        if (t.i64(nitf)) {
            if (nitf < 0) return bad("invalid InterfaceCount");
            for (long long i = 0; i < 5 * nitf; ++i) {
                long long v;
                if (!t.i64(v)) return bad("invalid interface line " + std::to_string(i / 5));
                itf_raw.push_back(v);
            }
        } else {
            // no interface list: consecutive domains touch at their last and
            // first elements (DBEM1/multidomain.cpp:1462-1474)
            itf_raw.push_back(-1);
        }
    }
    // model
    const std::string model = dir + "input/" + c.title + ".model";
    const std::string bdfile = dir + "input/" + c.title + ".bd";
    const bool model_bin = input_mode == 1 || (input_mode == 2 && file_exists(model + ".bin"));
    tdbem_status st = model_bin ? read_model_binary(model + ".bin", c) : read_model_text(model, c);
    if (st != TDBEM_OK) return st;
    const int64_t E = (int64_t)(c.elements.size() / 8);
    // materials (defaults: the card material) and interfaces
    c.n_domains = (int32_t)ndom;
    for (long long d = 0; d < ndom; ++d) c.materials.insert(c.materials.end(), {c.card_E, c.card_nu, c.card_rho});
    bool mat_zero = false;
    for (long long id : mid) mat_zero |= id == 0;
    for (size_t i = 0; i < mid.size(); ++i) {
        const int d = normalize_domain(mid[i], (int)ndom, mat_zero);
        if (d < 0) return bad("invalid domain material id " + std::to_string(mid[i]));
        for (int q = 0; q < 3; ++q) c.materials[3 * (size_t)d + q] = mval[3 * i + q];
    }
    if (!itf_raw.empty() && itf_raw[0] == -1 && itf_raw.size() == 1) {
        for (long long d = 0; d + 1 < ndom; ++d) {
            const int64_t base = E / ndom, extra = E % ndom;
            int64_t begin = 0;
            for (long long q = 0; q <= d; ++q) begin += base + (q < extra ? 1 : 0);
            c.interfaces.insert(c.interfaces.end(), {d, begin - 1, d + 1, begin, -1});
        }
    } else {
        bool ele_zero = false, dom_zero = false;
        for (size_t i = 0; i < itf_raw.size(); i += 5) {
            ele_zero |= itf_raw[i + 1] == 0 || itf_raw[i + 3] == 0;
            dom_zero |= itf_raw[i] == 0 || itf_raw[i + 2] == 0;
        }
        for (size_t i = 0; i < itf_raw.size(); i += 5) {
            const long long dA = normalize_domain(itf_raw[i], (int)ndom, dom_zero);
            const long long dB = normalize_domain(itf_raw[i + 2], (int)ndom, dom_zero);
            const long long eA = normalize_element(itf_raw[i + 1], E, ele_zero);
            const long long eB = normalize_element(itf_raw[i + 3], E, ele_zero);
            c.interfaces.insert(c.interfaces.end(),
                                {(int64_t)dA, (int64_t)eA, (int64_t)dB, (int64_t)eB,
                                 itf_raw[i + 4] == 0 ? -1 : (int64_t)itf_raw[i + 4]});
        }
    }
    // boundary values: the case's own .bd, or one load case per batch file
    const size_t per = (size_t)(c.n_steps + 1) * E * 3;
    if (batch_files.empty()) {
        c.n_loads = 1;
        c.known.resize(per);
        const bool bd_bin = input_mode == 1 || (input_mode == 2 && file_exists(bdfile + ".bin"));
        st = read_bd(bd_bin ? bdfile + ".bin" : bdfile, bd_bin, E, c.n_steps, c.bcid, nullptr, c.known.data());
        if (st != TDBEM_OK) return st;
    } else {
        c.n_loads = (int32_t)batch_files.size();
        c.known.resize(per * batch_files.size());
        for (size_t i = 0; i < batch_files.size(); ++i) {
            std::string p = batch_files[i];
            if (!p.empty() && p[0] != '/') p = dir + p;
            const bool b = p.size() > 4 && p.compare(p.size() - 4, 4, ".bin") == 0;
            st = read_bd(p, b, E, c.n_steps, c.bcid, i ? &c.bcid : nullptr, c.known.data() + per * i);
            if (st != TDBEM_OK) return st;
        }
    }
    *out = new tdbem_case(std::move(c));
    return TDBEM_OK;
}

tdbem_status tdbem_case_problem(const tdbem_case* c, tdbem_problem* p)
{
    if (!c || !p) return bad("null argument");
    *p = tdbem_problem{};
    p->n_points = (int64_t)(c->points.size() / 3);
    p->points = c->points.data();
    p->n_elements = (int64_t)(c->elements.size() / 8);
    p->elements = c->elements.data();
    p->bcid = c->bcid.data();
    p->n_domains = c->n_domains;
    p->materials = c->materials.data();
    p->n_interfaces = (int64_t)(c->interfaces.size() / 5);
    p->interfaces = c->interfaces.data();
    p->card_E = c->card_E;
    p->card_nu = c->card_nu;
    p->card_rho = c->card_rho;
    p->beta = c->beta;
    p->gap = c->gap;
    p->n_steps = c->n_steps;
    p->restart = c->restart;
    p->tol = c->tol;
    p->max_leaf = c->max_leaf;
    p->max_length = 1000.0;  // the reference driver's MaxLength (DBEM1/DBEM.cpp:1195)
    p->precision = TDBEM_PRECISION_FP64;
    p->n_loads = c->n_loads;
    return TDBEM_OK;
}

tdbem_status tdbem_case_known(const tdbem_case* c, double* known)
{
    if (!c || !known) return bad("null argument");
    std::memcpy(known, c->known.data(), sizeof(double) * c->known.size());
    return TDBEM_OK;
}

const char* tdbem_case_title(const tdbem_case* c) { return c ? c->title.c_str() : ""; }

void tdbem_case_destroy(tdbem_case* c) { delete c; }

}  // extern "C"
