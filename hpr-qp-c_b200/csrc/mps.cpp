// build_from_mps: free-format MPS / QPS reader (reference include/hprqp.h:31,
// src/shared/mps_qp.cpp:229-326 and src/shared/mps_reader.cpp).
//
// The accepted language and its meaning follow the reference reader so that
// a file gives the same HPRQPModel in both libraries:
//   * sections NAME, OBJSENSE (MIN; MAX is rejected), ROWS (N/E/L/G; the
//     first N row is the objective, later N rows are ignored), COLUMNS (one
//     or two row/value pairs per line, integer MARKER blocks), RHS (the
//     objective row's RHS is minus the objective constant), RANGES (E rows
//     widen towards the sign of the range, L/G rows get |range|), BOUNDS
//     (LO UP FX FR MI PL BV LI UI), QUADOBJ (one triangle, mirrored) or
//     QMATRIX (the full symmetric matrix), ENDATA;
//   * only the first RHS / RANGES / BOUNDS set name is used, lines of other
//     sets are skipped with a warning;
//   * default bounds [0, inf); a variable with only an upper bound u gets
//     lower bound -inf when u < 0, else 0; a variable with only a lower bound
//     gets upper bound inf;
//   * numbers may use a Fortran 'D' exponent; names are free-format tokens;
//   * duplicate (row, column) entries are summed.
//   * QCMATRIX <row> blocks (after COLUMNS, one per constraint row) give
//     x'Hx for that row; like the reference's file loader only diagonal H
//     is accepted, on one-sided rows, convex in the row's sense; such rows
//     become second-order cones through build_from_QAbc_qc_diagonal
//     (qcqp.cpp), the other rows keep their order.
// Discrete variables (integer markers, BV/LI/UI bounds) and maximisation are
// rejected with HPRQP_STATUS_INVALID_ARGUMENT like the reference.
//
// The implementation is this project's: a line tokenizer over std::string
// views, hash maps for names, COO triplets sorted stably into CSR, then the
// same builder as build_from_QAbc (model.cpp).
#include "hprqp.h"
#include "shared/qcqp.h"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

enum class Sec { None, Objsense, Rows, Columns, Rhs, Ranges, Bounds, Quad, Qcmatrix };
enum class RowKind { E, L, G };

constexpr size_t kMaxLine = 1022;   // longer lines are rejected
constexpr size_t kMaxToken = 255;   // longer names / numbers are rejected

struct Triplet {
    int row, col;
    double v;
};

struct Reader {
    // rows: index 0 = objective, -1 = ignored extra objective, 1.. = constraints
    std::unordered_map<std::string, int> rows;
    std::unordered_map<std::string, int> cols;
    std::vector<RowKind> kind;
    std::vector<double> lo_row, up_row;
    std::vector<double> c, lo_var, up_var;
    std::vector<char> discrete;
    std::vector<Triplet> a, q;
    std::vector<std::vector<std::pair<size_t, double>>> qc;  // per constraint row: (column, x'Hx coefficient)
    int qc_row = -1;                                          // row of the current QCMATRIX block
    double c0 = 0.0;
    bool have_obj = false, maximize = false, full_q = false, quadratic_rows = false;
    std::string rhs_set, rng_set, bnd_set;
    bool have_rhs_set = false, have_rng_set = false, have_bnd_set = false;
    long line_no = 0;

    bool fail(const char *what)
    {
        fprintf(stderr, "hprqp-b200: MPS line %ld: %s\n", line_no, what);
        return false;
    }
};

// strtod after mapping a Fortran 'D' exponent; the whole token must parse to a
// finite value
bool parse_number(const std::string &tok, double *out)
{
    std::string t(tok);
    for (char &ch : t)
        if (ch == 'd' || ch == 'D') ch = 'e';
    char *end = nullptr;
    errno = 0;
    const double v = strtod(t.c_str(), &end);
    if (end == t.c_str() || *end != '\0' || !std::isfinite(v) || errno == ERANGE) return false;
    *out = v;
    return true;
}

void split(const char *line, std::vector<std::string> &tok)
{
    tok.clear();
    const char *p = line;
    while (*p) {
        while (*p == ' ' || *p == '\t') ++p;
        if (!*p) break;
        const char *q = p;
        while (*q && *q != ' ' && *q != '\t') ++q;
        tok.emplace_back(p, (size_t)(q - p));
        p = q;
    }
}

// one (row, value) pair of a COLUMNS line
bool column_entry(Reader &R, int col, const std::string &rowname, double v)
{
    auto it = R.rows.find(rowname);
    if (it == R.rows.end()) return R.fail("unknown row in COLUMNS");
    if (it->second == 0) R.c[col] += v;
    else if (it->second > 0) R.a.push_back({it->second - 1, col, v});
    return true;
}

bool rhs_entry(Reader &R, const std::string &rowname, double v)
{
    auto it = R.rows.find(rowname);
    if (it == R.rows.end()) return R.fail("unknown row in RHS");
    if (it->second == 0) {
        R.c0 = -v;
    } else if (it->second < 0) {
        fprintf(stderr, "hprqp-b200: MPS line %ld: RHS of an ignored objective row skipped\n", R.line_no);
    } else {
        const int r = it->second - 1;
        if (R.kind[r] == RowKind::E) R.lo_row[r] = R.up_row[r] = v;
        else if (R.kind[r] == RowKind::L) R.up_row[r] = v;
        else R.lo_row[r] = v;
    }
    return true;
}

bool range_entry(Reader &R, const std::string &rowname, double v)
{
    auto it = R.rows.find(rowname);
    if (it == R.rows.end()) return R.fail("unknown row in RANGES");
    if (it->second <= 0) return R.fail("objective row in RANGES");
    const int r = it->second - 1;
    if (R.kind[r] == RowKind::E) {
        if (v >= 0.0) R.up_row[r] += v;
        else R.lo_row[r] += v;
    } else if (R.kind[r] == RowKind::L) {
        R.lo_row[r] = R.up_row[r] - std::fabs(v);
    } else {
        R.up_row[r] = R.lo_row[r] + std::fabs(v);
    }
    return true;
}

bool data_line(Reader &R, Sec sec, const std::vector<std::string> &t, bool &integer_block)
{
    const size_t nf = t.size();
    double v1 = 0.0, v2 = 0.0;
    const bool marker = sec == Sec::Columns && nf >= 2 && t[1] == "'MARKER'";
    if ((sec == Sec::Columns || sec == Sec::Rhs || sec == Sec::Ranges || sec == Sec::Quad) && !marker) {
        if ((nf != 3 && nf != 5) || (sec == Sec::Quad && nf != 3) || !parse_number(t[2], &v1) ||
            (nf == 5 && !parse_number(t[4], &v2)))
            return R.fail("invalid coefficient");
    }
    switch (sec) {
    case Sec::Objsense:
        if (t[0] == "MIN") R.maximize = false;
        else if (t[0] == "MAX") R.maximize = true;
        else return R.fail("unrecognised objective sense");
        return true;
    case Sec::Rows: {
        if (nf != 2 || (t[0] != "N" && t[0] != "E" && t[0] != "L" && t[0] != "G"))
            return R.fail("invalid ROWS entry");
        if (t[0] == "N") {
            if (!R.have_obj) {
                R.have_obj = true;
                R.rows[t[1]] = 0;
            } else {
                fprintf(stderr, "hprqp-b200: MPS line %ld: extra objective row %s ignored\n", R.line_no,
                        t[1].c_str());
                R.rows[t[1]] = -1;
            }
            return true;
        }
        if (R.rows.count(t[1])) return R.fail("duplicate row name");
        R.rows[t[1]] = (int)R.kind.size() + 1;
        const RowKind k = t[0] == "E" ? RowKind::E : (t[0] == "L" ? RowKind::L : RowKind::G);
        R.kind.push_back(k);
        R.lo_row.push_back(k == RowKind::L ? -INFINITY : 0.0);
        R.up_row.push_back(k == RowKind::G ? INFINITY : 0.0);
        return true;
    }
    case Sec::Columns: {
        if (marker) {
            if (nf >= 3 && t[2] == "'INTORG'") integer_block = true;
            else if (nf >= 3 && t[2] == "'INTEND'") integer_block = false;
            else return R.fail("unknown marker");
            return true;
        }
        auto it = R.cols.find(t[0]);
        int col;
        if (it == R.cols.end()) {
            col = (int)R.c.size();
            R.cols.emplace(t[0], col);
            R.c.push_back(0.0);
            R.lo_var.push_back(NAN);
            R.up_var.push_back(NAN);
            R.discrete.push_back(integer_block ? 1 : 0);
        } else {
            col = it->second;
        }
        if (!column_entry(R, col, t[1], v1)) return false;
        if (nf == 5 && !column_entry(R, col, t[3], v2)) return false;
        return true;
    }
    case Sec::Rhs:
        if (!R.have_rhs_set) {
            R.rhs_set = t[0];
            R.have_rhs_set = true;
        } else if (R.rhs_set != t[0]) {
            fprintf(stderr, "hprqp-b200: MPS line %ld: second RHS set %s skipped\n", R.line_no, t[0].c_str());
            return true;
        }
        if (!rhs_entry(R, t[1], v1)) return false;
        if (nf == 5 && !rhs_entry(R, t[3], v2)) return false;
        return true;
    case Sec::Ranges:
        if (!R.have_rng_set) {
            R.rng_set = t[0];
            R.have_rng_set = true;
        } else if (R.rng_set != t[0]) {
            fprintf(stderr, "hprqp-b200: MPS line %ld: second RANGES set %s skipped\n", R.line_no, t[0].c_str());
            return true;
        }
        if (!range_entry(R, t[1], v1)) return false;
        if (nf == 5 && !t[3].empty() && !range_entry(R, t[3], v2)) return false;
        return true;
    case Sec::Bounds: {
        double bv = 0.0;
        if (nf < 3 || nf > 4 || (nf == 4 && !parse_number(t[3], &bv))) return R.fail("invalid bound");
        if (!R.have_bnd_set) {
            R.bnd_set = t[1];
            R.have_bnd_set = true;
        } else if (R.bnd_set != t[1]) {
            fprintf(stderr, "hprqp-b200: MPS line %ld: second BOUNDS set %s skipped\n", R.line_no, t[1].c_str());
            return true;
        }
        auto it = R.cols.find(t[2]);
        if (it == R.cols.end()) return R.fail("unknown column in BOUNDS");
        const int j = it->second;
        const std::string &ty = t[0];
        if (ty == "FR") {
            R.lo_var[j] = -INFINITY;
            R.up_var[j] = INFINITY;
        } else if (ty == "MI") {
            R.lo_var[j] = -INFINITY;
        } else if (ty == "PL") {
            R.up_var[j] = INFINITY;
        } else if (ty == "BV") {
            R.discrete[j] = 1;
            R.lo_var[j] = 0.0;
            R.up_var[j] = 1.0;
        } else {
            if (nf < 4) return R.fail("bound needs a value");
            if (ty == "LO") {
                R.lo_var[j] = bv;
            } else if (ty == "UP") {
                R.up_var[j] = bv;
            } else if (ty == "FX") {
                R.lo_var[j] = R.up_var[j] = bv;
            } else if (ty == "LI") {
                R.discrete[j] = 1;
                R.lo_var[j] = bv;
            } else if (ty == "UI") {
                R.discrete[j] = 1;
                R.up_var[j] = bv;
            } else {
                return R.fail("unknown bound type");
            }
        }
        return true;
    }
    case Sec::Quad: {
        auto i1 = R.cols.find(t[0]), i2 = R.cols.find(t[1]);
        if (i1 == R.cols.end() || i2 == R.cols.end()) return R.fail("unknown column in the quadratic section");
        R.q.push_back({i1->second, i2->second, v1});
        return true;
    }
    case Sec::Qcmatrix: {
        // reference src/shared/mps_reader.cpp:968-990
        if (nf != 3 || !parse_number(t[2], &v1)) return R.fail("invalid QCMATRIX coefficient");
        auto i1 = R.cols.find(t[0]), i2 = R.cols.find(t[1]);
        if (i1 == R.cols.end() || i2 == R.cols.end()) return R.fail("unknown column in QCMATRIX");
        if (i1->second != i2->second && v1 != 0.0)
            return R.fail("non-diagonal QCMATRIX entries are not supported by the MPS reader; use "
                          "build_from_QAbc_qc_factors with a factor of the matrix");
        if (v1 != 0.0) R.qc[(size_t)R.qc_row].push_back({(size_t)i1->second, v1});
        return true;
    }
    default:
        return R.fail("data outside a section");
    }
}

// COO -> CSR, rows then columns ascending, duplicates summed in file order
void to_csr(size_t nrow, size_t ncol, const std::vector<Triplet> &t, std::vector<size_t> &rp,
            std::vector<size_t> &ci, std::vector<double> &v)
{
    std::vector<size_t> ord(t.size());
    std::iota(ord.begin(), ord.end(), size_t(0));
    std::stable_sort(ord.begin(), ord.end(), [&](size_t x, size_t y) {
        return t[x].row != t[y].row ? t[x].row < t[y].row : t[x].col < t[y].col;
    });
    rp.assign(nrow + 1, 0);
    ci.clear();
    v.clear();
    for (size_t k = 0; k < ord.size(); ++k) {
        const Triplet &e = t[ord[k]];
        if (k > 0 && e.row == t[ord[k - 1]].row && e.col == t[ord[k - 1]].col) {
            v.back() += e.v;
            continue;
        }
        ci.push_back((size_t)e.col);
        v.push_back(e.v);
        rp[(size_t)e.row + 1] += 1;
    }
    for (size_t r = 0; r < nrow; ++r) rp[r + 1] += rp[r];
    (void)ncol;
}

bool read_file(const char *path, Reader &R)
{
    FILE *fp = fopen(path, "r");
    if (!fp) {
        fprintf(stderr, "hprqp-b200: cannot open MPS file %s\n", path);
        return false;
    }
    std::vector<std::string> tok;
    char buf[kMaxLine + 2];
    Sec sec = Sec::None;
    bool seen_name = false, seen_objsense = false, seen_rows = false, seen_cols = false, seen_rhs = false,
         seen_bnd = false, seen_rng = false, seen_quad = false, ended = false, integer_block = false;
    std::vector<char> qc_rows;
    bool ok = true;
    while (ok && fgets(buf, sizeof buf, fp)) {
        ++R.line_no;
        if (!strchr(buf, '\n') && !feof(fp)) {
            ok = R.fail("line too long");
            break;
        }
        buf[strcspn(buf, "\r\n")] = '\0';
        if (buf[0] == '\0' || buf[0] == '*' || buf[0] == '&') continue;
        split(buf, tok);
        if (tok.empty()) continue;
        for (const auto &s : tok)
            if (s.size() > kMaxToken) {
                ok = R.fail("field too long");
                break;
            }
        if (!ok) break;
        if (buf[0] != ' ' && buf[0] != '\t') {
            const std::string &h = tok[0];
            const bool two = h == "NAME" || h == "OBJSENSE" || h == "QCMATRIX";
            if (two && tok.size() > 2) {
                ok = R.fail("too many fields in section header");
                break;
            }
            if (h == "NAME") {
                if (seen_name) ok = R.fail("second NAME section");
                seen_name = true;
            } else if (h == "OBJSENSE") {
                if (seen_objsense) ok = R.fail("second OBJSENSE section");
                seen_objsense = true;
                sec = Sec::Objsense;
                if (ok && tok.size() == 2) ok = data_line(R, sec, {tok[1]}, integer_block);
            } else if (h == "ROWS") {
                if (seen_rows) ok = R.fail("second ROWS section");
                seen_rows = true;
                sec = Sec::Rows;
            } else if (h == "COLUMNS") {
                if (seen_cols) ok = R.fail("second COLUMNS section");
                else if (!seen_rows) ok = R.fail("COLUMNS before ROWS");
                seen_cols = true;
                sec = Sec::Columns;
            } else if (h == "RHS") {
                if (seen_rhs) ok = R.fail("second RHS section");
                else if (!seen_rows || !seen_cols) ok = R.fail("RHS before ROWS and COLUMNS");
                seen_rhs = true;
                sec = Sec::Rhs;
            } else if (h == "BOUNDS") {
                if (seen_bnd) ok = R.fail("second BOUNDS section");
                else if (!seen_cols) ok = R.fail("BOUNDS before COLUMNS");
                seen_bnd = true;
                sec = Sec::Bounds;
            } else if (h == "RANGES") {
                if (seen_rng) ok = R.fail("second RANGES section");
                else if (!seen_rows || !seen_cols) ok = R.fail("RANGES before ROWS and COLUMNS");
                seen_rng = true;
                sec = Sec::Ranges;
            } else if (h == "QUADOBJ" || h == "QMATRIX") {
                if (seen_quad) ok = R.fail("second quadratic objective section");
                else if (!seen_cols) ok = R.fail("quadratic objective before COLUMNS");
                seen_quad = true;
                R.full_q = h == "QMATRIX";
                sec = Sec::Quad;
            } else if (h == "QCMATRIX") {
                auto it = tok.size() == 2 ? R.rows.find(tok[1]) : R.rows.end();
                if (!seen_cols || it == R.rows.end() || it->second <= 0) {
                    ok = R.fail("QCMATRIX needs a constraint row name after COLUMNS");
                } else {
                    if (qc_rows.empty()) qc_rows.assign(R.kind.size(), 0);
                    if (qc_rows[it->second - 1]) ok = R.fail("second QCMATRIX block for a row");
                    qc_rows[it->second - 1] = 1;
                    R.quadratic_rows = true;
                    if (R.qc.empty()) R.qc.resize(R.kind.size());
                    R.qc_row = it->second - 1;
                }
                sec = Sec::Qcmatrix;
            } else if (h == "ENDATA") {
                ended = true;
                break;
            } else {
                ok = R.fail("unsupported section");
            }
            continue;
        }
        if (tok.size() > 6) {
            ok = R.fail("too many fields");
            break;
        }
        ok = data_line(R, sec, tok, integer_block);
    }
    fclose(fp);
    if (ok && !ended) ok = R.fail("end of file before ENDATA");
    return ok;
}

// Quadratic rows (reference src/shared/mps_qp.cpp:119-206).  Each row's
// entries are sorted by (column, value), equal columns summed in that order,
// zeros dropped; a row left empty stays linear.  Otherwise the row must be
// one-sided: AL = -inf (sign +1) or AU = +inf (sign -1); D = 2 sign H must
// be >= 0 and finite; C = sign a_r; constant = -AU (sign +1) or AL (sign
// -1).  Returns false when no row is quadratic (the caller builds a QP).
bool build_quadratic_rows(const Reader &R, const HPRQPMatrixCSR *Q, const std::vector<size_t> &arp,
                          const std::vector<size_t> &aci, const std::vector<double> &av, const double *c,
                          const double *l, const double *u, HPRQPModel *model, HPRQPStatus *status)
{
    const size_t m = R.kind.size(), n = R.c.size();
    std::vector<std::vector<std::pair<size_t, double>>> diag(m);
    std::vector<double> sign(m, 1.0);
    size_t nq = 0;
    for (size_t r = 0; r < m && r < R.qc.size(); ++r) {
        auto d = R.qc[r];
        std::sort(d.begin(), d.end());
        size_t w = 0;
        for (const auto &e : d) {
            if (w && d[w - 1].first == e.first) d[w - 1].second += e.second;
            else d[w++] = e;
        }
        d.resize(w);
        d.erase(std::remove_if(d.begin(), d.end(), [](const std::pair<size_t, double> &e) { return e.second == 0.0; }),
                d.end());
        if (d.empty()) continue;
        const double lo = R.lo_row[r], up = R.up_row[r];
        if (lo == -INFINITY && std::isfinite(up)) sign[r] = 1.0;
        else if (up == INFINITY && std::isfinite(lo)) sign[r] = -1.0;
        else {
            fprintf(stderr, "hprqp-b200: a QCMATRIX row needs a one-sided inequality (not an equality, range or "
                            "free row)\n");
            *status = HPRQP_STATUS_INVALID_ARGUMENT;
            return true;
        }
        for (auto &e : d) {
            e.second *= 2.0 * sign[r];
            if (!std::isfinite(e.second) || e.second < 0.0) {
                fprintf(stderr, "hprqp-b200: a QCMATRIX row is not convex in its inequality sense\n");
                *status = HPRQP_STATUS_INVALID_ARGUMENT;
                return true;
            }
        }
        diag[r] = std::move(d);
        ++nq;
    }
    if (nq == 0) return false;
    std::vector<size_t> lrp(1, 0), lci, crp(1, 0), cci, drp(1, 0), dci;
    std::vector<double> lv, cv, dv, constant, al, au;
    for (size_t r = 0; r < m; ++r) {
        if (diag[r].empty()) {
            for (size_t k = arp[r]; k < arp[r + 1]; ++k) {
                lci.push_back(aci[k]);
                lv.push_back(av[k]);
            }
            lrp.push_back(lci.size());
            al.push_back(R.lo_row[r]);
            au.push_back(R.up_row[r]);
        } else {
            for (size_t k = arp[r]; k < arp[r + 1]; ++k) {
                cci.push_back(aci[k]);
                cv.push_back(sign[r] * av[k]);
            }
            crp.push_back(cci.size());
            for (const auto &e : diag[r]) {
                dci.push_back(e.first);
                dv.push_back(e.second);
            }
            drp.push_back(dci.size());
            constant.push_back(sign[r] > 0.0 ? -R.up_row[r] : R.lo_row[r]);
        }
    }
    size_t zi = 0;
    double zv = 0.0;
    auto pi = [&zi](std::vector<size_t> &x) { return x.empty() ? &zi : x.data(); };
    auto pv = [&zv](std::vector<double> &x) { return x.empty() ? &zv : x.data(); };
    HPRQPMatrixCSR lin{lrp.size() - 1, n, lci.size(), lrp.data(), pi(lci), pv(lv), 0};
    HPRQPMatrixCSR C{nq, n, cci.size(), crp.data(), pi(cci), pv(cv), 0};
    HPRQPMatrixCSR D{nq, n, dci.size(), drp.data(), pi(dci), pv(dv), 0};
    *status = build_from_QAbc_qc_diagonal(Q, &lin, c, al.empty() ? nullptr : al.data(),
                                          au.empty() ? nullptr : au.data(), l, u, R.c0, &C, constant.data(), &D,
                                          model);
    return true;
}

}  // namespace

extern "C" HPRQPStatus build_from_mps(const char *mps_path, HPRQPModel *model)
{
    if (!mps_path || !model) return HPRQP_STATUS_INVALID_ARGUMENT;
    model_init(model);
    Reader R;
    if (!read_file(mps_path, R)) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (R.maximize) {
        fprintf(stderr, "hprqp-b200: maximisation MPS input is not supported; give a convex minimisation\n");
        return HPRQP_STATUS_INVALID_ARGUMENT;
    }
    const size_t n = R.c.size(), m = R.kind.size();
    // default and one-sided variable bounds
    for (size_t j = 0; j < n; ++j) {
        double &l = R.lo_var[j], &u = R.up_var[j];
        if (std::isnan(l) && std::isnan(u)) {
            l = 0.0;
            u = R.discrete[j] ? 1.0 : INFINITY;
        } else if (std::isnan(l)) {
            l = u < 0.0 ? -INFINITY : 0.0;
        } else if (std::isnan(u)) {
            u = INFINITY;
        }
    }
    for (size_t j = 0; j < n; ++j)
        if (R.discrete[j]) {
            fprintf(stderr, "hprqp-b200: discrete MPS variables are not supported\n");
            return HPRQP_STATUS_INVALID_ARGUMENT;
        }
    std::vector<size_t> arp, aci, qrp, qci;
    std::vector<double> av, qv;
    to_csr(m, n, R.a, arp, aci, av);
    if (!R.full_q) {
        // one triangle given: mirror the off-diagonal entries
        const size_t q0 = R.q.size();
        for (size_t k = 0; k < q0; ++k)
            if (R.q[k].row != R.q[k].col) R.q.push_back({R.q[k].col, R.q[k].row, R.q[k].v});
    }
    to_csr(n, n, R.q, qrp, qci, qv);
    if (R.full_q) {
        // the full matrix must be exactly symmetric
        for (size_t i = 0; i < n; ++i)
            for (size_t k = qrp[i]; k < qrp[i + 1]; ++k) {
                const size_t j = qci[k];
                auto b = qci.begin() + (long)qrp[j], e = qci.begin() + (long)qrp[j + 1];
                auto it = std::lower_bound(b, e, i);
                const double other = (it != e && *it == i) ? qv[(size_t)(it - qci.begin())] : 0.0;
                if (other != qv[k]) {
                    fprintf(stderr, "hprqp-b200: QMATRIX must hold a symmetric full matrix\n");
                    return HPRQP_STATUS_INVALID_ARGUMENT;
                }
            }
    }
    auto nz = [](std::vector<size_t> &x) { return x.empty() ? (size_t *)nullptr : x.data(); };
    auto nzd = [](std::vector<double> &x) { return x.empty() ? (double *)nullptr : x.data(); };
    double dummy_s = 0.0;
    size_t dummy_i = 0;
    HPRQPMatrixCSR Q{n, n, qv.size(), qrp.data(), qci.empty() ? &dummy_i : nz(qci), qv.empty() ? &dummy_s : nzd(qv), 0};
    HPRQPMatrixCSR A{m, n, av.size(), arp.data(), aci.empty() ? &dummy_i : nz(aci), av.empty() ? &dummy_s : nzd(av), 0};
    std::vector<double> cc(R.c), l(R.lo_var), u(R.up_var);
    double one = 0.0;
    if (R.quadratic_rows) {
        HPRQPStatus st = HPRQP_STATUS_OK;
        if (build_quadratic_rows(R, &Q, arp, aci, av, cc.empty() ? &one : cc.data(), l.empty() ? &one : l.data(),
                                 u.empty() ? &one : u.data(), model, &st))
            return st;
    }
    return build_from_QAbc(&Q, &A, cc.empty() ? &one : cc.data(), m ? R.lo_row.data() : nullptr,
                           m ? R.up_row.data() : nullptr, l.empty() ? &one : l.data(), u.empty() ? &one : u.data(),
                           R.c0, model);
}

// the reference's name for the same reader (include/shared/build.h;
// src/shared/mps_qp.cpp:208, which its build_from_mps calls)
extern "C" HPRQPStatus build_model_from_mps(const char *mps_path, HPRQPModel *model)
{
    return build_from_mps(mps_path, model);
}
