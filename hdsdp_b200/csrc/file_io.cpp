// SDPA sparse-format reader (host only), behind the reference's HReadSDPA
// (interface/hdsdp_file_io.h:7, interface/hdsdp_file_io.c:34-381).
//
// The file holds, after comment lines starting with '*' or '"': the number of
// constraints, the number of blocks, the block sizes (a negative last size is a
// diagonal LP block of that many columns), the right-hand side, then one entry per
// line "constraint block row column value" with 1-based block, row and column and
// constraint 0 standing for the objective matrix. Separators { } ( ) , in the size
// and right-hand-side lines are ignored. Parsing stops at the end of the file or at
// a "BEGIN.COMMENT" line; any other line that is not an entry (a blank line before
// the end included) is an error, as is an index out of range.
//
// Output, as the reference produces it: per SDP block a CSC matrix with PACK_NNZ(n)
// rows (packed lower triangle, PACK_IDX(n, i, j) = (2n - j - 1) j / 2 + i, i >= j) and
// nConstrs + 1 columns (column 0 the objective, negated); for the LP block a CSC
// matrix with nLPCols rows and nConstrs + 1 columns (column 0 negated). Entries with
// |value| < 1e-12 are dropped (one warning). Within a column entries keep file order
// and repeated positions are kept as separate entries. nCols is the sum of n^2 over the
// SDP blocks; nElems counts the entries kept. All arrays are malloc'ed; the caller
// frees them with free().
#include "../../include/hdsdp.h"
#include "../../include/hdsdp_file_io.h"

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

namespace {

struct Triplet {
    int row, col;
    double val;
};

// CSC arrays of `ncol` columns from triplets, entries of a column in input order.
void compress(const std::vector<Triplet> &t, int ncol, int **beg, int **idx, double **val) {
    *beg = (int *) calloc((size_t) ncol + 1, sizeof(int));
    *idx = (int *) calloc(t.empty() ? 1 : t.size(), sizeof(int));
    *val = (double *) calloc(t.empty() ? 1 : t.size(), sizeof(double));
    if (!*beg || !*idx || !*val) return;
    for (const Triplet &e : t) (*beg)[e.col + 1] += 1;
    for (int c = 0; c < ncol; ++c) (*beg)[c + 1] += (*beg)[c];
    std::vector<int> next((*beg), (*beg) + ncol);
    for (const Triplet &e : t) {
        const int at = next[e.col]++;
        (*idx)[at] = e.row;
        (*val)[at] = e.val;
    }
}

bool is_comment(const std::string &line) { return !line.empty() && (line[0] == '*' || line[0] == '"'); }

// Numbers of a header line, with { } ( ) , as separators.
std::vector<double> header_numbers(const std::string &line) {
    std::string s = line;
    for (char &ch : s)
        if (ch == '{' || ch == '}' || ch == '(' || ch == ')' || ch == ',') ch = ' ';
    std::vector<double> out;
    const char *p = s.c_str();
    char *end = nullptr;
    while (*p) {
        while (*p && std::isspace((unsigned char) *p)) ++p;
        if (!*p) break;
        const double v = std::strtod(p, &end);
        if (end == p) {
            ++p;  // skip a character that starts no number
            continue;
        }
        out.push_back(v);
        p = end;
    }
    return out;
}

bool read_line(FILE *f, std::string &line) {
    line.clear();
    int ch;
    bool any = false;
    while ((ch = std::fgetc(f)) != EOF) {
        any = true;
        if (ch == '\n') break;
        line.push_back((char) ch);
    }
    if (!line.empty() && line.back() == '\r') line.pop_back();
    return any;
}

}  // namespace

extern "C" hdsdp_retcode HReadSDPA(char *fname, int *pnConstrs, int *pnBlks, int **pblkDims, double **prowRHS,
                                   int ***pconeMatBeg, int ***pconeMatIdx, double ***pconeMatElem, int *pnCols,
                                   int *pnLPCols, int **pLpMatBeg, int **pLpMatIdx, double **pLpMatElem,
                                   int *pnElems) {
    if (!fname) return HDSDP_RETCODE_FAILED;
    FILE *f = std::fopen(fname, "r");
    if (!f) return HDSDP_RETCODE_FAILED;
    std::string line;
    auto fail = [&](hdsdp_retcode r) {
        std::fclose(f);
        return r;
    };
    // comments, then the constraint count and the block count, one per line
    bool got = false;
    while ((got = read_line(f, line)) && (line.empty() || is_comment(line))) {
    }
    if (!got) return fail(HDSDP_RETCODE_FAILED);
    std::vector<double> v = header_numbers(line);
    if (v.empty()) return fail(HDSDP_RETCODE_FAILED);
    const int nConstrs = (int) v[0];
    if (!read_line(f, line)) return fail(HDSDP_RETCODE_FAILED);
    v = header_numbers(line);
    if (v.empty()) return fail(HDSDP_RETCODE_FAILED);
    int nBlocks = (int) v[0];
    if (nConstrs < 0 || nBlocks <= 0) return fail(HDSDP_RETCODE_FAILED);
    // block sizes (may run over several lines); only the last may be negative (LP)
    std::vector<int> sizes;
    while ((int) sizes.size() < nBlocks) {
        if (!read_line(f, line)) return fail(HDSDP_RETCODE_FAILED);
        for (double d : header_numbers(line)) {
            if ((int) sizes.size() < nBlocks) sizes.push_back((int) d);
        }
    }
    int nLPCols = 0, nSDP = nBlocks;
    for (int b = 0; b < nBlocks; ++b) {
        if (sizes[b] == 0) return fail(HDSDP_RETCODE_FAILED);
        if (sizes[b] < 0) {
            if (b != nBlocks - 1) return fail(HDSDP_RETCODE_FAILED);
            nLPCols = -sizes[b];
            nSDP = nBlocks - 1;
        }
    }
    // right-hand side (may run over several lines)
    std::vector<double> rhs;
    while ((int) rhs.size() < nConstrs) {
        if (!read_line(f, line)) return fail(HDSDP_RETCODE_FAILED);
        for (double d : header_numbers(line))
            if ((int) rhs.size() < nConstrs) rhs.push_back(d);
    }
    // entries
    std::vector<std::vector<Triplet>> sdp(nSDP);
    std::vector<Triplet> lp;
    long nElems = 0;
    bool warned = false;
    while (read_line(f, line)) {
        int con, blk, i, j;
        double val;
        if (std::sscanf(line.c_str(), "%d %d %d %d %lg", &con, &blk, &i, &j, &val) != 5) {
            // as in the reference: the end of the data is a "BEGIN.COMMENT" line or a last
            // line without a newline; any other line that is not an entry is an error
            if (std::strncmp(line.c_str(), "BEGIN.COMMENT", 13) == 0 || std::feof(f)) break;
            return fail(HDSDP_RETCODE_FAILED);
        }
        if (con < 0 || con > nConstrs || blk < 1 || blk > nBlocks) return fail(HDSDP_RETCODE_FAILED);
        const int b = blk - 1;
        int r = i - 1, c = j - 1;
        if (std::fabs(val) < 1e-12) {
            if (!warned) {
                std::printf("[Warning] Entry smaller than 1e-12 is ignored. \n");
                warned = true;
            }
            continue;
        }
        if (con == 0) val = -val;
        if (nLPCols > 0 && b == nBlocks - 1) {
            if (r < 0 || r >= nLPCols) return fail(HDSDP_RETCODE_FAILED);
            lp.push_back({r, con, val});
        } else {
            const int n = sizes[b];
            if (r > c) std::swap(r, c);  // r <= c: the packed entry is row c, column r
            if (r < 0 || c >= n) return fail(HDSDP_RETCODE_FAILED);
            const int packed = (int) ((2LL * n - r - 1) * r / 2 + c);
            sdp[b].push_back({packed, con, val});
        }
        nElems += 1;
    }
    std::fclose(f);

    // outputs
    int *dims = (int *) calloc((size_t) (nSDP > 0 ? nSDP : 1), sizeof(int));
    double *b = (double *) calloc((size_t) (nConstrs > 0 ? nConstrs : 1), sizeof(double));
    int **beg = (int **) calloc((size_t) (nSDP > 0 ? nSDP : 1), sizeof(int *));
    int **idx = (int **) calloc((size_t) (nSDP > 0 ? nSDP : 1), sizeof(int *));
    double **elem = (double **) calloc((size_t) (nSDP > 0 ? nSDP : 1), sizeof(double *));
    if (!dims || !b || !beg || !idx || !elem) return HDSDP_RETCODE_MEMORY;
    int nCols = 0;
    for (int k = 0; k < nSDP; ++k) {
        dims[k] = sizes[k];
        nCols += sizes[k] * sizes[k];
        compress(sdp[k], nConstrs + 1, &beg[k], &idx[k], &elem[k]);
        if (!beg[k] || !idx[k] || !elem[k]) return HDSDP_RETCODE_MEMORY;
    }
    for (int k = 0; k < nConstrs; ++k) b[k] = rhs[k];
    int *lbeg = nullptr, *lidx = nullptr;
    double *lval = nullptr;
    if (nLPCols > 0) {
        compress(lp, nConstrs + 1, &lbeg, &lidx, &lval);
        if (!lbeg || !lidx || !lval) return HDSDP_RETCODE_MEMORY;
    }
    *pnConstrs = nConstrs;
    *pnBlks = nSDP;
    *pblkDims = dims;
    *prowRHS = b;
    *pconeMatBeg = beg;
    *pconeMatIdx = idx;
    *pconeMatElem = elem;
    *pnCols = nCols;
    *pnLPCols = nLPCols;
    *pLpMatBeg = lbeg;
    *pLpMatIdx = lidx;
    *pLpMatElem = lval;
    *pnElems = (int) nElems;
    return HDSDP_RETCODE_OK;
}
