// mtx.cu -- the on-disk boundary: MatrixMarket export and import of a
// BCOO system, in the formats the reference writes and reads
// (GlobalLinearSystem::export_matrix_market_files,
// SG/linear_system/linear_system/global_linear_system.cu:98-261;
// read_mm_coordinate_real / read_mm_array_vector_mx1 /
// to_upper_triangle_block_triplets, SG/main.cu:398-646), so systems the
// reference dumps can be replayed here and the other way round.  Host code.
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <strings.h>

#include <algorithm>
#include <array>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/sgmas.h"
#include "ctx.hpp"

namespace {

struct File {
    FILE* f;
    explicit File(const char* path, const char* mode) : f(fopen(path, mode)) {}
    ~File() { if (f) fclose(f); }
};

// "%%MatrixMarket matrix <format> <field> <symmetry>", tokens compared
// without case; returns false on anything else
bool read_banner(FILE* f, std::string& format, std::string& field, std::string& symmetry) {
    char line[1100];
    if (!fgets(line, sizeof(line), f)) return false;
    char b[64], obj[64], fmt[64], fld[64], sym[64];
    if (sscanf(line, "%63s %63s %63s %63s %63s", b, obj, fmt, fld, sym) != 5) return false;
    if (strcmp(b, "%%MatrixMarket") != 0 || strcasecmp(obj, "matrix") != 0) return false;
    auto lower = [](const char* s) { std::string t(s); for (auto& ch : t) ch = (char)tolower(ch); return t; };
    format = lower(fmt);
    field = lower(fld);
    symmetry = lower(sym);
    return true;
}

// first non-comment line
bool next_data_line(FILE* f, char* line, int n) {
    while (fgets(line, n, f))
        if (line[0] != '%') return true;
    return false;
}

}  // namespace

extern "C" int sgmas_mtx_write(const char* path_A, const char* path_b, const double* values, const int* rows,
                               const int* cols, int n_blocks, int n_block_rows, const double* b) {
    if (!path_A || n_blocks < 0 || n_block_rows < 1 || (n_blocks > 0 && (!values || !rows || !cols)) ||
        (path_b && !b))
        return SGMAS_ERR_ARG;
    const int M = 3 * n_block_rows;
    if (path_b) {
        File fb(path_b, "w");
        if (!fb.f) return ctx_fail(nullptr, SGMAS_ERR_ARG, "cannot open %s for writing", path_b);
        fprintf(fb.f, "%%%%MatrixMarket matrix array real general\n%d %d\n", M, 1);
        for (int i = 0; i < M; ++i) fprintf(fb.f, "%.17g\n", b[i]);
        if (ferror(fb.f)) return ctx_fail(nullptr, SGMAS_ERR_ARG, "write error on %s", path_b);
    }
    long long nnz = 0;
    for (int k = 0; k < n_blocks; ++k) nnz += rows[k] == cols[k] ? 9 : 18;
    if (nnz > 0x7fffffffLL) return ctx_fail(nullptr, SGMAS_ERR_CAPACITY, "A has more than 2^31-1 entries");
    File fa(path_A, "w");
    if (!fa.f) return ctx_fail(nullptr, SGMAS_ERR_ARG, "cannot open %s for writing", path_A);
    fprintf(fa.f, "%%%%MatrixMarket matrix coordinate real general\n%d %d %d\n", M, M, (int)nnz);
    for (int k = 0; k < n_blocks; ++k) {
        const int bi = rows[k], bj = cols[k];
        const double* B = values + 9 * (size_t)k;  // column-major: (i, j) at i + 3 j
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) fprintf(fa.f, "%d %d %.17g\n", 3 * bi + i + 1, 3 * bj + j + 1, B[i + 3 * j]);
        if (bi != bj)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    fprintf(fa.f, "%d %d %.17g\n", 3 * bj + i + 1, 3 * bi + j + 1, B[j + 3 * i]);
    }
    if (ferror(fa.f)) return ctx_fail(nullptr, SGMAS_ERR_ARG, "write error on %s", path_A);
    return SGMAS_OK;
}

extern "C" int sgmas_mtx_read(const char* path_A, const char* path_b, double* values, int* rows, int* cols,
                              int cap_blocks, double* b, int cap_b, int* n_blocks, int* n_block_rows) {
    if (!path_A || !n_blocks || !n_block_rows) return SGMAS_ERR_ARG;
    File fa(path_A, "r");
    if (!fa.f) return ctx_fail(nullptr, SGMAS_ERR_ARG, "cannot open %s", path_A);
    std::string fmt, fld, sym;
    if (!read_banner(fa.f, fmt, fld, sym) || fmt != "coordinate" || fld != "real")
        return ctx_fail(nullptr, SGMAS_ERR_ARG, "%s: need a MatrixMarket coordinate real matrix", path_A);
    const bool symmetric = sym == "symmetric";
    char line[1100];
    int M = 0, N = 0, nz = 0;
    if (!next_data_line(fa.f, line, sizeof(line)) || sscanf(line, "%d %d %d", &M, &N, &nz) != 3)
        return ctx_fail(nullptr, SGMAS_ERR_ARG, "%s: bad size line", path_A);
    if (M != N || M % 3 != 0 || nz < 0)
        return ctx_fail(nullptr, SGMAS_ERR_ARG, "%s: A must be square with 3x3 blocks (M=%d N=%d)", path_A, M, N);
    const int nb = M / 3;
    // blocks accumulated in file order, upper triangle at the block level
    std::unordered_map<uint64_t, std::array<double, 9>> blocks;
    blocks.reserve((size_t)nz / 4 + 16);
    std::vector<char> diag(nb, 0);
    for (int k = 0; k < nz; ++k) {
        int r, c;
        double v;
        if (fscanf(fa.f, "%d %d %lg", &r, &c, &v) != 3)
            return ctx_fail(nullptr, SGMAS_ERR_ARG, "%s: entry %d unreadable", path_A, k);
        --r;
        --c;
        if (r < 0 || c < 0 || r >= M || c >= N)
            return ctx_fail(nullptr, SGMAS_ERR_ARG, "%s: entry %d out of range", path_A, k);
        int bi = r / 3, bj = c / 3, li = r % 3, lj = c % 3;
        if (bi > bj) {
            if (!symmetric) continue;  // the expanded lower triangle of a general file
            std::swap(bi, bj);
            std::swap(li, lj);
        }
        auto it = blocks.try_emplace(((uint64_t)bi << 32) | (uint32_t)bj, std::array<double, 9>{}).first;
        it->second[li + 3 * lj] += v;
        if (symmetric && bi == bj && li != lj) it->second[lj + 3 * li] += v;
        if (bi == bj) diag[bi] = 1;
    }
    for (int i = 0; i < nb; ++i)
        if (!diag[i]) return ctx_fail(nullptr, SGMAS_ERR_ARG, "%s: diagonal block %d missing", path_A, i);
    std::vector<uint64_t> keys;
    keys.reserve(blocks.size());
    for (const auto& kv : blocks) keys.push_back(kv.first);
    std::sort(keys.begin(), keys.end());
    *n_blocks = (int)keys.size();
    *n_block_rows = nb;
    int nbv = 0;
    File fb(path_b ? path_b : "", "r");
    if (path_b) {
        if (!fb.f) return ctx_fail(nullptr, SGMAS_ERR_ARG, "cannot open %s", path_b);
        if (!read_banner(fb.f, fmt, fld, sym) || fmt != "array" || fld != "real")
            return ctx_fail(nullptr, SGMAS_ERR_ARG, "%s: need a MatrixMarket array real matrix", path_b);
        int bm = 0, bn = 0;
        if (!next_data_line(fb.f, line, sizeof(line)) || sscanf(line, "%d %d", &bm, &bn) != 2 || bn != 1)
            return ctx_fail(nullptr, SGMAS_ERR_ARG, "%s: b must be an M x 1 array", path_b);
        if (bm != M) return ctx_fail(nullptr, SGMAS_ERR_ARG, "%s: b has %d rows, A has %d", path_b, bm, M);
        nbv = bm;
    }
    if (!values || !rows || !cols || cap_blocks < *n_blocks || (path_b && (!b || cap_b < nbv)))
        return SGMAS_ERR_CAPACITY;  // sizes are in *n_blocks / *n_block_rows: call again with room
    for (size_t k = 0; k < keys.size(); ++k) {
        rows[k] = (int)(keys[k] >> 32);
        cols[k] = (int)(keys[k] & 0xffffffffu);
        memcpy(values + 9 * k, blocks[keys[k]].data(), 9 * sizeof(double));
    }
    for (int i = 0; i < nbv; ++i)
        if (fscanf(fb.f, "%lg", &b[i]) != 1) return ctx_fail(nullptr, SGMAS_ERR_ARG, "%s: entry %d unreadable", path_b, i);
    return SGMAS_OK;
}
