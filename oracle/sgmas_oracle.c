/*
 * sgmas_oracle.c -- CPU restatement of StiffGIPC's MAS-PCG Newton-step solve.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Loaded by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU legs; never by the product
 * path.  Each function restates the reference file:line named in its comment
 * (paths relative to the StiffGIPC project, "SG/" = StiffGIPC/).
 *
 * Ordering conventions for floating-point sums (the reference uses atomics,
 * so its own order is not defined):
 *   - MAS component sums of the residual: member lanes in ascending order;
 *   - Schwarz products: columns ascending, each 3x3 row an fma chain;
 *   - CollectFinalZ: level order, as the reference;
 *   - Gauss-Jordan inverse: exactly the reference's per-element operation
 *     sequence (IEEE divide, fused multiply-add), so it is bit-reproducible.
 */
#include "sgmas_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_MAX_LEVELS 6

static int round_up(int v, int b) { return (v + b - 1) / b * b; }
static unsigned lanemask_lt(int lane) { return (lane >= 32) ? 0xffffffffu : ((1u << lane) - 1u); }
static int ffs0(unsigned v) { return __builtin_ffs((int)v) - 1; }
static int popc(unsigned v) { return __builtin_popcount(v); }

int or_omp_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* setMAS_partition (SG/main.cu:47-75) after load_parts (SG/load_mesh.cpp:   */
/* 449-480: part_offset = last part id + 1).                                 */
/* Returns 0, or a negative code where the reference would write out of      */
/* bounds (-2: a part has more than `bank` vertices) or leave real_map       */
/* entries unset (-3: parts not contiguous in vertex order).                 */
/* ------------------------------------------------------------------------ */
int or_mas_partition(const int* part_id, int n, int bank, int* part_offset_out,
                     int* part_map, int part_map_cap, int* real_map)
{
    if(n < 1 || bank < 1 || bank > 32)
        return -1;
    int part_offset = part_id[n - 1] + 1;
    int size        = part_offset * bank;
    if(part_offset < 1 || size > part_map_cap)
        return -1;
    for(int i = 0; i < size; i++)
        part_map[i] = -1;
    int index = 0;
    for(int i = 0; i < n; i++)
    {
        if(part_id[i] < 0 || part_id[i] >= part_offset || index >= bank)
            return -2;
        part_map[bank * part_id[i] + index] = i;
        index++;
        if(i <= n - 2 && part_id[i + 1] != part_id[i])
            index = 0;
    }
    index = 0;
    for(int i = 0; i < size; i++)
    {
        if(part_map[i] == index)
        {
            real_map[index] = i;
            index++;
        }
    }
    if(part_offset_out)
        *part_offset_out = part_offset;
    return index == n ? 0 : -3;
}

/* ------------------------------------------------------------------------ */
/* tetrahedra_obj::getVertNeighbors (SG/load_mesh.cpp:894-999).  Edges are  */
/* kept in the orientation first inserted, iterated in std::set<pair> order. */
/* ------------------------------------------------------------------------ */
typedef struct { uint64_t a, b; int64_t seq; } or_edge;

static int cmp_undirected(const void* x, const void* y)
{
    const or_edge* e = (const or_edge*)x;
    const or_edge* f = (const or_edge*)y;
    uint64_t e0 = e->a < e->b ? e->a : e->b, e1 = e->a < e->b ? e->b : e->a;
    uint64_t f0 = f->a < f->b ? f->a : f->b, f1 = f->a < f->b ? f->b : f->a;
    if(e0 != f0) return e0 < f0 ? -1 : 1;
    if(e1 != f1) return e1 < f1 ? -1 : 1;
    return (e->seq < f->seq) ? -1 : (e->seq > f->seq);
}
static int cmp_directed(const void* x, const void* y)
{
    const or_edge* e = (const or_edge*)x;
    const or_edge* f = (const or_edge*)y;
    if(e->a != f->a) return e->a < f->a ? -1 : 1;
    if(e->b != f->b) return e->b < f->b ? -1 : 1;
    return 0;
}

int or_vert_neighbors(const int* tets, int ntet, const int* tris, int ntri,
                      int n_verts, int abd_vert_offset, unsigned* nb_start,
                      unsigned* nb_num, unsigned* nb_list, int nb_cap)
{
    if(n_verts <= 0)
        return 0;
    int64_t cand = 6LL * ntet + 9LL * ntri;
    or_edge* E   = (or_edge*)malloc(sizeof(or_edge) * (cand > 0 ? cand : 1));
    int64_t  m   = 0;
    static const int tp[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
    for(int t = 0; t < ntet; t++)
        for(int k = 0; k < 6; k++)
        {
            E[m].a   = (uint64_t)(uint32_t)tets[4 * t + tp[k][0]];
            E[m].b   = (uint64_t)(uint32_t)tets[4 * t + tp[k][1]];
            E[m].seq = m;
            m++;
        }
    for(int t = 0; t < ntri; t++)
        for(int rep = 0; rep < 3; rep++) /* the reference loops i < 3 over the same three edges */
        {
            uint32_t x = (uint32_t)tris[3 * t], y = (uint32_t)tris[3 * t + 1],
                     z = (uint32_t)tris[3 * t + 2];
            E[m].a = x; E[m].b = y; E[m].seq = m; m++;
            E[m].a = y; E[m].b = z; E[m].seq = m; m++;
            E[m].a = z; E[m].b = x; E[m].seq = m; m++;
        }
    qsort(E, (size_t)m, sizeof(or_edge), cmp_undirected);
    int64_t u = 0;
    for(int64_t i = 0; i < m; i++)
    {
        if(i > 0)
        {
            uint64_t p0 = E[u - 1].a < E[u - 1].b ? E[u - 1].a : E[u - 1].b;
            uint64_t p1 = E[u - 1].a < E[u - 1].b ? E[u - 1].b : E[u - 1].a;
            uint64_t c0 = E[i].a < E[i].b ? E[i].a : E[i].b;
            uint64_t c1 = E[i].a < E[i].b ? E[i].b : E[i].a;
            if(p0 == c0 && p1 == c1)
                continue;
        }
        E[u++] = E[i];
    }
    qsort(E, (size_t)u, sizeof(or_edge), cmp_directed);
    for(int i = 0; i < n_verts; i++)
        nb_num[i] = 0;
    for(int64_t i = 0; i < u; i++)
    {
        int64_t f = (int64_t)E[i].a - abd_vert_offset, s = (int64_t)E[i].b - abd_vert_offset;
        if(f < 0 || f >= n_verts || s < 0 || s >= n_verts)
        {
            free(E);
            return -1;
        }
        nb_num[f]++;
        nb_num[s]++;
    }
    unsigned off = 0;
    for(int i = 0; i < n_verts; i++)
    {
        nb_start[i] = off;
        off += nb_num[i];
    }
    if((int64_t)off > nb_cap)
    {
        free(E);
        return -2;
    }
    unsigned* fill = (unsigned*)calloc((size_t)n_verts, sizeof(unsigned));
    for(int64_t i = 0; i < u; i++)
    {
        int64_t f = (int64_t)E[i].a - abd_vert_offset, s = (int64_t)E[i].b - abd_vert_offset;
        nb_list[nb_start[f] + fill[f]++] = (unsigned)s;
        nb_list[nb_start[s] + fill[s]++] = (unsigned)f;
    }
    free(fill);
    free(E);
    return (int)off;
}

/* MASPreconditioner::computeNumLevels (SG/MASPreconditioner.cu:1720-1739). */
int or_num_levels(int max_nodes, int bank)
{
    int nLevel  = 1;
    int levelSz = round_up(max_nodes, bank);
    while(levelSz > bank)
    {
        levelSz /= bank;
        nLevel++;
        levelSz = round_up(levelSz, bank);
    }
    nLevel = nLevel + 1;
    return nLevel > OR_MAX_LEVELS ? OR_MAX_LEVELS : nLevel;
}

/* ------------------------------------------------------------------------ */
/* Morton codes: expand_bits / hash_code(type=-1) (SG/GIPC.cu:142-168) and   */
/* _calcVertMChash (SG/GIPC.cu:412-461) with the AABB of the vertices.       */
/* ------------------------------------------------------------------------ */
static uint32_t expand_bits(uint32_t v)
{
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
static double clampd(double x, double lo, double hi)
{
    /* std::min(std::max(x, lo), hi) with std:: argument order semantics */
    double t = (x < lo) ? lo : x;
    return (hi < t) ? hi : t;
}
static uint32_t to_u32(double v)
{
    /* the GPU conversion (cvt.rzi.u32.f64) maps NaN to 0 */
    if(!(v == v))
        return 0u;
    return (uint32_t)v;
}
uint32_t or_hash_code(double x, double y, double z, double resolution)
{
    x = clampd(x * resolution, 0.0, resolution - 1.0);
    y = clampd(y * resolution, 0.0, resolution - 1.0);
    z = clampd(z * resolution, 0.0, resolution - 1.0);
    uint32_t xx = expand_bits(to_u32(x));
    uint32_t yy = expand_bits(to_u32(y));
    uint32_t zz = expand_bits(to_u32(z));
    return (xx << 2) + (yy << 1) + zz;
}
void or_vert_morton(const double* pos, int n, uint64_t* out)
{
    if(n < 1)
        return;
    double lo[3] = {pos[0], pos[1], pos[2]}, hi[3] = {pos[0], pos[1], pos[2]};
    for(int i = 1; i < n; i++)
        for(int d = 0; d < 3; d++)
        {
            if(pos[3 * i + d] < lo[d]) lo[d] = pos[3 * i + d];
            if(pos[3 * i + d] > hi[d]) hi[d] = pos[3 * i + d];
        }
    double sz[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    for(int i = 0; i < n; i++)
    {
        uint64_t mc32 = or_hash_code((pos[3 * i] - lo[0]) / sz[0],
                                     (pos[3 * i + 1] - lo[1]) / sz[1],
                                     (pos[3 * i + 2] - lo[2]) / sz[2], 1024.0);
        out[i] = (mc32 << 32) | (uint64_t)(uint32_t)i;
    }
}

/* ------------------------------------------------------------------------ */
/* Spmv::warp_reduce_sym_spmv (SG/linear_system/utils/spmv.cu:8-133):        */
/* y = a*A*x + b*y over upper 3x3 blocks (column-major values).              */
/* ------------------------------------------------------------------------ */
void or_spmv_sym(double a, const double* vals, const int* rows, const int* cols,
                 int nb, const double* x, double b, double* y, int ndof)
{
    for(int i = 0; i < ndof; i++)
        y[i] = (b != 0) ? b * y[i] : 0.0;
    for(int k = 0; k < nb; k++)
    {
        const double* H = vals + 9 * (size_t)k;
        int i = rows[k], j = cols[k];
        for(int r = 0; r < 3; r++)
        {
            double s = H[r] * x[3 * j] + H[r + 3] * x[3 * j + 1] + H[r + 6] * x[3 * j + 2];
            y[3 * i + r] += a * s;
        }
        if(i != j)
            for(int r = 0; r < 3; r++)
            {
                double s = H[3 * r] * x[3 * i] + H[3 * r + 1] * x[3 * i + 1] + H[3 * r + 2] * x[3 * i + 2];
                y[3 * j + r] += a * s;
            }
    }
}

double or_dot(const double* a, const double* b, int n)
{
    double s = 0;
    for(int i = 0; i < n; i++)
        s += a[i] * b[i];
    return s;
}

/* ------------------------------------------------------------------------ */
/* Converter::convert (SG/linear_system/utils/converter.cu:23-189): stable   */
/* sort by key (row<<32)+col, then sum equal keys.  The sum runs in the      */
/* stable sorted order.                                                      */
/* ------------------------------------------------------------------------ */
typedef struct { uint64_t key; int idx; } or_key;
static int cmp_key(const void* x, const void* y)
{
    const or_key* a = (const or_key*)x;
    const or_key* b = (const or_key*)y;
    if(a->key != b->key) return a->key < b->key ? -1 : 1;
    return (a->idx > b->idx) - (a->idx < b->idx);
}
int or_convert(const double* vals, const int* rows, const int* cols, int n,
               double* out_vals, int* out_rows, int* out_cols)
{
    if(n < 1)
        return 0;
    or_key* K = (or_key*)malloc(sizeof(or_key) * (size_t)n);
    for(int i = 0; i < n; i++)
    {
        K[i].key = ((uint64_t)(uint32_t)rows[i] << 32) + (uint64_t)(uint32_t)cols[i];
        K[i].idx = i;
    }
    qsort(K, (size_t)n, sizeof(or_key), cmp_key);
    int u = -1;
    for(int i = 0; i < n; i++)
    {
        if(i == 0 || K[i].key != K[i - 1].key)
        {
            u++;
            out_rows[u] = (int)(K[i].key >> 32);
            out_cols[u] = (int)(K[i].key & 0xffffffffu);
            memcpy(out_vals + 9 * (size_t)u, vals + 9 * (size_t)K[i].idx, 9 * sizeof(double));
        }
        else
        {
            for(int q = 0; q < 9; q++)
                out_vals[9 * (size_t)u + q] += vals[9 * (size_t)K[i].idx + q];
        }
    }
    free(K);
    return u + 1;
}

/* write_triplet_fem (SG/femEnergy.cu:14-62): the upper 3x3 blocks of a     */
/* (3*nnode)^2 row-major element matrix, swapped+transposed when row > col. */
void or_write_upper_blocks(const double* H, int nnode, const int* nodes,
                           double* vals, int* rows, int* cols)
{
    int kk = 0, w = 3 * nnode;
    for(int ii = 0; ii < nnode; ii++)
        for(int jj = ii; jj < nnode; jj++)
        {
            int row = nodes[ii], col = nodes[jj];
            int swap = row > col;
            rows[kk] = swap ? col : row;
            cols[kk] = swap ? row : col;
            for(int a = 0; a < 3; a++)
                for(int c = 0; c < 3; c++)
                    vals[9 * kk + a + 3 * c] = swap ? H[(jj * 3 + a) * w + ii * 3 + c]
                                                    : H[(ii * 3 + a) * w + jj * 3 + c];
            kk++;
        }
}

/* ------------------------------------------------------------------------ */
/* MAS preconditioner (SG/MASPreconditioner.cu).                             */
/* ------------------------------------------------------------------------ */
struct or_mas
{
    int bank, N, Mm, levelnum, total, node_offset;
    int nb_size, gn_cap;
    unsigned *nb_list0, *nb_num0, *nb_start, *nb_list, *nb_num;
    int *part_map, *real_map;
    unsigned* fine_mask;
    unsigned* next_mask;
    int* prefix_orig;
    int* coarse_space;
    int* going_next;
    int level_size[2 * (OR_MAX_LEVELS + 2)];
    int* coarse_table; /* N x 6 */
    /* matrices */
    int nblk, bsym, precision;
    double* hess;  /* nblk x bsym x 9 (col-major 3x3) */
    double* inv64;
    float*  inv32;
};

static void* xcalloc(size_t n, size_t s) { return calloc(n ? n : 1, s); }

or_mas* or_mas_create(int bank, int n_verts, int collision_node_offset,
                      const unsigned* nb_list, int nb_size, const unsigned* nb_start,
                      const unsigned* nb_num, const int* part_map, int part_map_size,
                      const int* real_map)
{
    if(bank != 16 && bank != 32)
        return NULL;
    if(n_verts < 1 || part_map_size < n_verts || part_map_size % bank)
        return NULL;
    or_mas* m      = (or_mas*)calloc(1, sizeof(or_mas));
    m->bank        = bank;
    m->N           = n_verts;
    m->Mm          = part_map_size;
    m->node_offset = collision_node_offset;
    int maxNodes   = part_map_size > n_verts ? part_map_size : n_verts;
    m->levelnum    = or_num_levels(maxNodes, bank);
    m->nb_size     = nb_size;
    m->nb_list0    = (unsigned*)xcalloc((size_t)nb_size, sizeof(unsigned));
    m->nb_list     = (unsigned*)xcalloc((size_t)nb_size, sizeof(unsigned));
    memcpy(m->nb_list0, nb_list, sizeof(unsigned) * (size_t)nb_size);
    m->nb_num0  = (unsigned*)xcalloc((size_t)n_verts, sizeof(unsigned));
    m->nb_num   = (unsigned*)xcalloc((size_t)n_verts, sizeof(unsigned));
    m->nb_start = (unsigned*)xcalloc((size_t)n_verts, sizeof(unsigned));
    memcpy(m->nb_num0, nb_num, sizeof(unsigned) * (size_t)n_verts);
    memcpy(m->nb_start, nb_start, sizeof(unsigned) * (size_t)n_verts);
    m->part_map = (int*)xcalloc((size_t)part_map_size, sizeof(int));
    m->real_map = (int*)xcalloc((size_t)n_verts, sizeof(int));
    memcpy(m->part_map, part_map, sizeof(int) * (size_t)part_map_size);
    memcpy(m->real_map, real_map, sizeof(int) * (size_t)n_verts);
    m->fine_mask    = (unsigned*)xcalloc((size_t)n_verts, sizeof(unsigned));
    m->next_mask    = (unsigned*)xcalloc((size_t)n_verts, sizeof(unsigned));
    m->prefix_orig  = (int*)xcalloc((size_t)(part_map_size / bank), sizeof(int));
    m->coarse_space = (int*)xcalloc((size_t)n_verts * m->levelnum, sizeof(int));
    /* goingNext holds level-0 entries by vertex id and level>=1 entries by
     * global node id; every level adds at most N nodes plus padding. */
    m->gn_cap       = round_up(part_map_size, bank) + (m->levelnum + 1) * (n_verts + bank);
    m->going_next   = (int*)xcalloc((size_t)m->gn_cap, sizeof(int));
    m->coarse_table = (int*)xcalloc((size_t)n_verts * 6, sizeof(int));
    return m;
}

void or_mas_destroy(or_mas* m)
{
    if(!m)
        return;
    free(m->nb_list0); free(m->nb_list); free(m->nb_num0); free(m->nb_num);
    free(m->nb_start); free(m->part_map); free(m->real_map); free(m->fine_mask);
    free(m->next_mask); free(m->prefix_orig); free(m->coarse_space);
    free(m->going_next); free(m->coarse_table); free(m->hess); free(m->inv64);
    free(m->inv32);
    free(m);
}

int or_mas_levelnum(const or_mas* m) { return m->levelnum; }
int or_mas_total_clusters(const or_mas* m) { return m->total; }

/* Decode one contact int4 into its vertex list
 * (_buildCollisionConnection_new, SG/MASPreconditioner.cu:1126-1538). */
static int decode_pair(const int* p, int v[4])
{
    int x = p[0], y = p[1], z = p[2], w = p[3];
    if(x >= 0)
    {
        if(w < 0) w = -w - 1;
        v[0] = x; v[1] = y; v[2] = z; v[3] = w;
        return 4;
    }
    x = -x - 1;
    if(z < 0)
    {
        if(y < 0)
        {
            v[0] = x; v[1] = -y - 1; v[2] = -z - 1; v[3] = -w - 1;
            return 4;
        }
        v[0] = x; v[1] = y;
        return 2;
    }
    if(w < 0)
    {
        if(y < 0)
        {
            v[0] = x; v[1] = -y - 1; v[2] = z; v[3] = -w - 1;
            return 4;
        }
        v[0] = x; v[1] = y; v[2] = z;
        return 3;
    }
    v[0] = x; v[1] = y; v[2] = z; v[3] = w;
    return 4;
}

/* _buildCollisionConnection_new: OR same-bank bits between the nodes of one
 * contact; level < 1 uses the slot map and ORs into fine_mask[vertex],
 * level >= 1 uses the coarse table and ORs into mask[coarse id]. */
static void collision_connection(or_mas* m, unsigned* mask, int level, const int* pairs, int cp)
{
    int b = m->bank;
    for(int q = 0; q < cp; q++)
    {
        int v[4], id[4];
        unsigned cm[4] = {0, 0, 0, 0};
        int nv = decode_pair(pairs + 4 * q, v);
        for(int i = 0; i < nv; i++)
        {
            v[i] -= m->node_offset;
            if(v[i] >= 0 && v[i] < m->N)
                id[i] = (level >= 1) ? m->coarse_space[(size_t)(level - 1) * m->N + v[i]]
                                     : m->real_map[v[i]];
            else
                id[i] = -1;
        }
        for(int i = 0; i < nv; i++)
            for(int j = i + 1; j < nv; j++)
            {
                if(id[i] == id[j] || id[i] < 0 || id[j] < 0)
                    continue;
                if(id[i] / b == id[j] / b)
                {
                    cm[i] |= 1u << (id[j] % b);
                    cm[j] |= 1u << (id[i] % b);
                }
            }
        for(int i = 0; i < nv; i++)
        {
            if(level >= 1)
            {
                if(id[i] >= 0)
                    mask[id[i]] |= cm[i];
            }
            else if(v[i] >= 0 && v[i] < m->N)
                mask[v[i]] |= cm[i];
        }
    }
}

/* Closure of one bank's masks and cluster count: the BFS of
 * _preparePrefixSumL0_new (:157-214) / _nextLevelCluster (:480-528). */
static void bank_closure(const unsigned* orig, const int* valid, int b, unsigned* out, int* count)
{
    int cnt = 0;
    for(int lane = 0; lane < b; lane++)
    {
        if(!valid[lane])
            continue;
        unsigned msk = orig[lane], visited = 1u << lane;
        for(;;)
        {
            unsigned todo = visited ^ msk;
            if(!todo)
                break;
            int nv = ffs0(todo);
            visited |= 1u << nv;
            msk |= orig[nv];
        }
        out[lane] = msk;
        if(popc(msk & lanemask_lt(lane)) == 0)
            cnt++;
    }
    *count = cnt;
}

/* MASPreconditioner::ReorderRealtime (SG/MASPreconditioner.cu:1768-1807). */
int or_mas_reorder(or_mas* m, const int* pairs4, int cp_num)
{
    const int b = m->bank, N = m->N, Mm = m->Mm, L = m->levelnum;
    const int nbank0 = Mm / b;
    /* neighbour lists are reset from their initial copies before every
     * rebuild (setPreconditioner_bcoo, :2179-2187) */
    memcpy(m->nb_list, m->nb_list0, sizeof(unsigned) * (size_t)m->nb_size);
    memcpy(m->nb_num, m->nb_num0, sizeof(unsigned) * (size_t)N);
    memset(m->level_size, 0, sizeof(m->level_size));

    /* _buildCML0_new (:63-103) */
    for(int tdx = 0; tdx < Mm; tdx++)
    {
        int idx = m->part_map[tdx];
        if(idx < 0)
            continue;
        int w = tdx / b, lane = tdx % b;
        unsigned msk = 1u << lane;
        unsigned nk = 0, st = m->nb_start[idx];
        for(unsigned i = 0; i < m->nb_num[idx]; i++)
        {
            unsigned vc = m->nb_list[st + i];
            int s       = m->real_map[vc];
            if(s / b == w)
                msk |= 1u << (s % b);
            else
                m->nb_list[st + nk++] = vc;
        }
        m->nb_num[idx]    = nk;
        m->fine_mask[idx] = msk;
    }
    if(cp_num > 0)
        collision_connection(m, m->fine_mask, -1, pairs4, cp_num);

    /* _preparePrefixSumL0_new (:157-214) */
    {
        unsigned orig[32], clo[32];
        int valid[32];
        for(int w = 0; w < nbank0; w++)
        {
            for(int lane = 0; lane < b; lane++)
            {
                int idx     = m->part_map[w * b + lane];
                valid[lane] = idx >= 0;
                orig[lane]  = idx >= 0 ? m->fine_mask[idx] : 0;
                clo[lane]   = 0;
            }
            int cnt;
            bank_closure(orig, valid, b, clo, &cnt);
            for(int lane = 0; lane < b; lane++)
                if(valid[lane])
                    m->fine_mask[m->part_map[w * b + lane]] = clo[lane];
            /* an all-padding bank is never written by the reference; 0 here */
            m->prefix_orig[w] = cnt;
        }
    }

    /* exclusive scan + _buildLevel1_new (:1592-1613, :271-328) */
    int* psum = (int*)xcalloc((size_t)nbank0, sizeof(int));
    for(int w = 1; w < nbank0; w++)
        psum[w] = psum[w - 1] + m->prefix_orig[w - 1];
    const int r16 = round_up(Mm, b);
    m->level_size[2 * 1 + 0] = psum[nbank0 - 1] + m->prefix_orig[nbank0 - 1];
    m->level_size[2 * 1 + 1] = r16;
    for(int w = 0; w < nbank0; w++)
    {
        unsigned elected = 0;
        for(int lane = 0; lane < b; lane++)
        {
            int idx = m->part_map[w * b + lane];
            if(idx >= 0 && popc(m->fine_mask[idx] & lanemask_lt(lane)) == 0)
                elected |= 1u << lane;
        }
        for(int lane = 0; lane < b; lane++)
        {
            int idx = m->part_map[w * b + lane];
            if(idx < 0)
                continue;
            int el                = ffs0(m->fine_mask[idx]);
            int id                = popc(elected & lanemask_lt(el)) + psum[w];
            m->coarse_space[idx]  = id;
            m->going_next[idx]    = id + r16;
        }
    }
    free(psum);

    for(int level = 1; level < L; level++)
    {
        memset(m->next_mask, 0, sizeof(unsigned) * (size_t)N);
        /* _buildConnectMaskLx_new (:401-477); the per-component OR of the
         * reference equals the per-vertex OR below because every member of a
         * level-0 component shares its coarse id at every level. */
        for(int tdx = 0; tdx < Mm; tdx++)
        {
            int idx = m->part_map[tdx];
            if(idx < 0)
                continue;
            int ci = m->coarse_space[(size_t)(level - 1) * N + idx];
            unsigned conn = 0, nk = 0, st = m->nb_start[idx];
            for(unsigned i = 0; i < m->nb_num[idx]; i++)
            {
                unsigned vc = m->nb_list[st + i];
                int cc      = m->coarse_space[(size_t)(level - 1) * N + vc];
                if(ci / b == cc / b)
                    conn |= 1u << (cc % b);
                else
                    m->nb_list[st + nk++] = vc;
            }
            m->nb_num[idx] = nk;
            m->next_mask[ci] |= conn;
        }
        if(cp_num > 0)
            collision_connection(m, m->next_mask, level, pairs4, cp_num);

        const int count = m->level_size[2 * level + 0];
        const int begin = m->level_size[2 * level + 1];
        if(count < 1)
            break;
        const int nbank = (count + b - 1) / b;
        int* np  = (int*)xcalloc((size_t)nbank, sizeof(int));
        int* nps = (int*)xcalloc((size_t)nbank, sizeof(int));
        unsigned* clo_all = (unsigned*)xcalloc((size_t)count, sizeof(unsigned));
        /* _nextLevelCluster (:480-528) */
        for(int w = 0; w < nbank; w++)
        {
            unsigned orig[32], clo[32];
            int valid[32];
            for(int lane = 0; lane < b; lane++)
            {
                int idx     = w * b + lane;
                valid[lane] = idx < count;
                orig[lane]  = idx < count ? ((1u << lane) | m->next_mask[idx]) : 0;
                clo[lane]   = 0;
            }
            int cnt;
            bank_closure(orig, valid, b, clo, &cnt);
            for(int lane = 0; lane < b && w * b + lane < count; lane++)
                clo_all[w * b + lane] = clo[lane];
            np[w] = cnt;
        }
        /* exclusive scan + _prefixSumLx (:1690-1706, :530-577) */
        for(int w = 1; w < nbank; w++)
            nps[w] = nps[w - 1] + np[w - 1];
        const int rc = round_up(count, b);
        m->level_size[2 * (level + 1) + 0] = nps[nbank - 1] + np[nbank - 1];
        m->level_size[2 * (level + 1) + 1] = begin + rc;
        for(int w = 0; w < nbank; w++)
        {
            unsigned elected = 0;
            for(int lane = 0; lane < b && w * b + lane < count; lane++)
                if(popc(clo_all[w * b + lane] & lanemask_lt(lane)) == 0)
                    elected |= 1u << lane;
            for(int lane = 0; lane < b && w * b + lane < count; lane++)
            {
                int idx = w * b + lane;
                int el  = ffs0(clo_all[idx]);
                int id  = popc(elected & lanemask_lt(el)) + nps[w];
                m->next_mask[idx] = (unsigned)id;
                if(idx + begin < m->gn_cap)
                    m->going_next[idx + begin] = id + begin + rc;
            }
        }
        /* _computeNextLevel (:579-590) */
        for(int v = 0; v < N; v++)
        {
            int nx = m->coarse_space[(size_t)(level - 1) * N + v];
            m->coarse_space[(size_t)level * N + v] = (int)m->next_mask[nx];
        }
        free(np); free(nps); free(clo_all);
    }
    m->total = m->level_size[2 * L + 1];

    /* _aggregationKernel (:592-625) */
    for(int v = 0; v < N; v++)
    {
        int cur = v;
        for(int l = 0; l < 6; l++)
            m->coarse_table[6 * (size_t)v + l] = 0;
        for(int l = 0; l < L - 1; l++)
        {
            int nx = m->going_next[cur];
            m->coarse_table[6 * (size_t)v + l] = nx;
            cur = nx;
        }
    }
    return m->total;
}

int or_mas_get_tables(const or_mas* m, unsigned* fine_mask, int* coarse_space,
                      int* going_next, int going_next_cap, int* level_size,
                      int* prefix_orig, int* coarse_table)
{
    if(fine_mask) memcpy(fine_mask, m->fine_mask, sizeof(unsigned) * (size_t)m->N);
    if(coarse_space) memcpy(coarse_space, m->coarse_space, sizeof(int) * (size_t)m->N * m->levelnum);
    if(going_next)
    {
        int n = going_next_cap < m->gn_cap ? going_next_cap : m->gn_cap;
        memcpy(going_next, m->going_next, sizeof(int) * (size_t)n);
    }
    if(level_size) memcpy(level_size, m->level_size, sizeof(int) * 2 * (size_t)(m->levelnum + 1));
    if(prefix_orig) memcpy(prefix_orig, m->prefix_orig, sizeof(int) * (size_t)(m->Mm / m->bank));
    if(coarse_table) memcpy(coarse_table, m->coarse_table, sizeof(int) * 6 * (size_t)m->N);
    return 0;
}

/* packed upper index of block (r, c), r <= c: SG/MASPreconditioner.cu:1857 */
static int sym_index(int b, int r, int c) { return b * r - r * (r + 1) / 2 + c; }

static double* blk(or_mas* m, int node_r, int node_c)
{
    /* nodes in the same bank, node_r%b <= node_c%b */
    int b = m->bank;
    return m->hess + ((size_t)(node_c / b) * m->bsym + sym_index(b, node_r % b, node_c % b)) * 9;
}
static void add3(double* D, const double* H, int transpose)
{
    for(int i = 0; i < 3; i++)
        for(int j = 0; j < 3; j++)
            D[i + 3 * j] += transpose ? H[j + 3 * i] : H[i + 3 * j];
}

/* Gauss-Jordan inverse of one expanded bank matrix, no pivoting:
 * __inverse6_P96x96 (SG/MASPreconditioner.cu:626-724). */
static void gj_invert(const double* packed, int b, double* out_packed)
{
    const int n = 3 * b;
    double* S   = (double*)malloc(sizeof(double) * (size_t)n * n);
    double* col = (double*)malloc(sizeof(double) * (size_t)n);
    for(int j = 0; j < n; j++)
        for(int i = 0; i < n; i++)
        {
            int rb = j / 3, cb = i / 3;
            double v;
            if(cb >= rb)
                v = packed[sym_index(b, rb, cb) * 9 + (j % 3) + 3 * (i % 3)];
            else
                v = packed[sym_index(b, cb, rb) * 9 + (i % 3) + 3 * (j % 3)];
            if(i == j && v == 0)
                v = 1;
            S[(size_t)j * n + i] = v;
        }
    for(int j = 0; j < n; j++)
    {
        double rt = S[(size_t)j * n + j];
        for(int i = 0; i < n; i++)
            col[i] = S[(size_t)i * n + j];
        for(int i = 0; i < n; i++)
            S[(size_t)i * n + j] = (i == j) ? 1.0 : 0.0;
        for(int i = 0; i < n; i++)
            S[(size_t)j * n + i] /= rt;
        for(int k = 0; k < n; k++)
        {
            if(k == j)
                continue;
            double rate = -col[k];
            for(int i = 0; i < n; i++)
                S[(size_t)k * n + i] = fma(rate, S[(size_t)j * n + i], S[(size_t)k * n + i]);
        }
    }
    /* partial symmetrisation of the diagonal 3x3 blocks (:705-708) */
    for(int i = 0; i < n; i++)
    {
        if(i % 3 < 2)
            S[(size_t)(i + 1) * n + i] = S[(size_t)i * n + i + 1];
        else
            S[(size_t)i * n + i - 2] = S[(size_t)(i - 2) * n + i];
    }
    for(int j = 0; j < n; j++)
        for(int i = 0; i < n; i++)
        {
            int rb = j / 3, cb = i / 3;
            if(cb >= rb)
                out_packed[sym_index(b, rb, cb) * 9 + (j % 3) + 3 * (i % 3)] = S[(size_t)j * n + i];
        }
    free(S);
    free(col);
}

/* Factored inverse (the library's storage for its BF16 and FP32-factored
 * MAS, not a reference kernel): lower Cholesky M = L L^T (right-looking, a
 * pivot that is not positive becomes 1, zero diagonal -> 1 as the reference's
 * inverse), then W = L^-1 column by column; slot (rb, cb), rb <= cb, of the
 * output holds block (cb, rb) of W, column-major.  M^-1 = W^T W.  Operation
 * order per element as the device kernel k_chol_inv. */
static void chol_factor(const double* packed, int b, double* out_packed)
{
    const int n = 3 * b;
    double* A  = (double*)calloc((size_t)n * n, sizeof(double));
    double* dW = (double*)malloc(sizeof(double) * (size_t)n);
    for(int i = 0; i < n; i++)
        for(int j = 0; j <= i; j++)
        {
            int rb = j / 3, cb = i / 3;
            double v = rb == cb ? packed[sym_index(b, rb, rb) * 9 + (i % 3) + 3 * (j % 3)]
                                : packed[sym_index(b, rb, cb) * 9 + (j % 3) + 3 * (i % 3)];
            if(i == j && v == 0)
                v = 1;
            A[(size_t)i * n + j] = v;
        }
    for(int k = 0; k < n; k++)
    {
        double d = A[(size_t)k * n + k];
        if(!(d > 0.0))
            d = 1.0;
        const double lkk = sqrt(d);
        for(int i = k + 1; i < n; i++)
            A[(size_t)i * n + k] = A[(size_t)i * n + k] / lkk;
        A[(size_t)k * n + k] = lkk;
        for(int i = k + 1; i < n; i++)
        {
            const double lik = A[(size_t)i * n + k];
            for(int j = k + 1; j <= i; j++)
                A[(size_t)i * n + j] = fma(-lik, A[(size_t)j * n + k], A[(size_t)i * n + j]);
        }
    }
    for(int j = 0; j < n; j++)
        dW[j] = 1.0 / A[(size_t)j * n + j];
    /* W_ij (i > j) = acc / L_ii with acc = +0 then acc = fma(-L_ik, W_kj, acc)
       for k = j .. i-1 ascending (W_jj = 1 / L_jj) */
    for(int j = 0; j < n; j++)
        for(int i = j + 1; i < n; i++)
        {
            double acc = 0.0;
            for(int k = j; k < i; k++)
                acc = fma(-A[(size_t)i * n + k], k == j ? dW[j] : A[(size_t)j * n + k], acc);
            A[(size_t)j * n + i] = acc / A[(size_t)i * n + i];
        }
    for(int rb = 0; rb < b; rb++)
        for(int cb = rb; cb < b; cb++)
            for(int q = 0; q < 9; q++)
            {
                int i = 3 * cb + q % 3, j = 3 * rb + q / 3;
                double v = i > j ? A[(size_t)j * n + i] : (i == j ? dW[i] : 0.0);
                out_packed[sym_index(b, rb, cb) * 9 + q] = v;
            }
    free(A);
    free(dW);
}

static int is_factored(int precision) { return precision == 1 || precision == 3; }

static void invert_one(const double* packed, int b, double* out_packed, int precision)
{
    if(is_factored(precision))
        chol_factor(packed, b, out_packed);
    else
        gj_invert(packed, b, out_packed);
}

void or_mas_invert_blocks(const double* in, int nblocks, int bank, double* out64)
{
    int bsym = bank * (bank + 1) / 2;
    for(int k = 0; k < nblocks; k++)
        gj_invert(in + (size_t)k * bsym * 9, bank, out64 + (size_t)k * bsym * 9);
}

int or_mas_factor_blocks(const double* in, int nblocks, int bank, double* out64)
{
    int bsym = bank * (bank + 1) / 2;
    for(int k = 0; k < nblocks; k++)
        chol_factor(in + (size_t)k * bsym * 9, bank, out64 + (size_t)k * bsym * 9);
    return 0;
}

static float bf16_round_f(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    if((u & 0x7f800000u) == 0x7f800000u)
    {
        if(u & 0x007fffffu)
            u = (u | 0x00400000u) & 0xffff0000u; /* quiet NaN */
        else
            u &= 0xffff0000u;
    }
    else
    {
        uint32_t lsb = (u >> 16) & 1u;
        u += 0x7fffu + lsb;
        u &= 0xffff0000u;
    }
    float r;
    memcpy(&r, &u, 4);
    return r;
}

int or_bf16_round(const double* in, int n, float* out)
{
    for(int i = 0; i < n; i++)
        out[i] = bf16_round_f((float)in[i]);
    return 0;
}

/* MASPreconditioner::setPreconditioner_bcoo + PrepareHessian_bcoo
 * (SG/MASPreconditioner.cu:2169-2207, :1810-2054) and the inverse.
 * Deliberate difference: a same-bank block whose column slot precedes its
 * row slot is stored transposed (the reference drops it at :1856; with the
 * reference's own slot maps that case cannot occur because slots follow
 * vertex order inside a bank). */
int or_mas_assemble(or_mas* m, const double* vals, const int* rows, const int* cols,
                    const uint32_t* indices, int offset, int n, int precision)
{
    const int b = m->bank, L = m->levelnum, N = m->N;
    if(m->total <= 0)
        return -1;
    m->nblk      = m->total / b;
    m->bsym      = b * (b + 1) / 2;
    m->precision = precision;
    size_t nval  = (size_t)m->nblk * m->bsym * 9;
    free(m->hess); free(m->inv64); free(m->inv32);
    m->hess  = (double*)xcalloc(nval, sizeof(double));
    m->inv64 = (double*)xcalloc(nval, sizeof(double));
    m->inv32 = (float*)xcalloc(nval, sizeof(float));

    /* phase 1: every FEM block */
    for(int I = 0; I < n; I++)
    {
        int k  = indices ? (int)indices[I] : I;
        int rr = rows[k] - offset, cc = cols[k] - offset;
        if(rr < 0 || rr >= N || cc < 0 || cc >= N)
            continue; /* not in the FEM range (calculate_subsystem_bcoo_indices) */
        const double* H = vals + 9 * (size_t)k;
        int sr = m->real_map[rr], sc = m->real_map[cc];
        if(sr / b == sc / b)
        {
            if(sc >= sr)
                memcpy(blk(m, sr, sc), H, 9 * sizeof(double));
            else
            {
                double* D = blk(m, sc, sr);
                for(int i = 0; i < 3; i++)
                    for(int j = 0; j < 3; j++)
                        D[i + 3 * j] = H[j + 3 * i];
            }
            continue;
        }
        int vr = rr, vc = cc;
        for(int level = 1; level < L; level++)
        {
            vr = m->going_next[vr];
            vc = m->going_next[vc];
            if(vr / b != vc / b)
                continue;
            if(vc >= vr)
            {
                add3(blk(m, vr, vc), H, 0);
                if(vc == vr)
                    add3(blk(m, vr, vc), H, 1);
            }
            else
                add3(blk(m, vc, vr), H, 1);
        }
    }
    /* phase 2: bank contents pushed to the coarser levels */
    const int nbank0 = m->Mm / b;
    for(int h = 0; h < nbank0; h++)
    {
        int prefix = m->prefix_orig[h];
        double S[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        int lead = -1;
        for(int r = 0; r < b; r++)
            for(int c = 0; c < b; c++)
            {
                int rdx = m->part_map[h * b + r], cdx = m->part_map[h * b + c];
                if(rdx < 0 || cdx < 0)
                    continue;
                double mat[9];
                if(c >= r)
                    memcpy(mat, m->hess + ((size_t)h * m->bsym + sym_index(b, r, c)) * 9, sizeof(mat));
                else
                {
                    const double* T = m->hess + ((size_t)h * m->bsym + sym_index(b, c, r)) * 9;
                    for(int i = 0; i < 3; i++)
                        for(int j = 0; j < 3; j++)
                            mat[i + 3 * j] = T[j + 3 * i];
                }
                if(prefix == 1)
                {
                    for(int q = 0; q < 9; q++)
                        S[q] += mat[q];
                    if(lead < 0)
                        lead = rdx;
                    continue;
                }
                int vr = rdx, vc = cdx;
                for(int level = 1; level < L; level++)
                {
                    vr = m->going_next[vr];
                    vc = m->going_next[vc];
                    if(vr / b == vc / b && vc >= vr)
                        add3(blk(m, vr, vc), mat, 0);
                }
            }
        if(prefix == 1 && lead >= 0)
        {
            int nx = m->going_next[lead];
            for(int level = 1; level < L; level++)
            {
                add3(blk(m, nx, nx), S, 0);
                nx = m->going_next[nx];
            }
        }
    }
    /* inverse, then storage precision */
#pragma omp parallel for schedule(dynamic, 4)
    for(int k = 0; k < m->nblk; k++)
        invert_one(m->hess + (size_t)k * m->bsym * 9, b, m->inv64 + (size_t)k * m->bsym * 9, precision);
    for(size_t i = 0; i < nval; i++)
    {
        float f     = (float)m->inv64[i];
        m->inv32[i] = (precision == 1) ? bf16_round_f(f) : f;
    }
    return 0;
}

/* Replace the assembled FP64 subdomain matrices (e.g. by the device's) and
 * recompute the inverses and their storage precision, so an apply can be
 * compared on identical matrices. */
int or_mas_set_hess(or_mas* m, const double* hess, int precision)
{
    if(!m->hess)
        return -1;
    size_t nval  = (size_t)m->nblk * m->bsym * 9;
    m->precision = precision;
    memcpy(m->hess, hess, nval * sizeof(double));
#pragma omp parallel for schedule(dynamic, 4)
    for(int k = 0; k < m->nblk; k++)
        invert_one(m->hess + (size_t)k * m->bsym * 9, m->bank, m->inv64 + (size_t)k * m->bsym * 9, precision);
    for(size_t i = 0; i < nval; i++)
    {
        float f     = (float)m->inv64[i];
        m->inv32[i] = (precision == 1) ? bf16_round_f(f) : f;
    }
    return 0;
}

int or_mas_get_matrices(const or_mas* m, double* hess64, double* inv64, float* inv32)
{
    size_t nval = (size_t)m->nblk * m->bsym * 9;
    if(hess64) memcpy(hess64, m->hess, nval * sizeof(double));
    if(inv64) memcpy(inv64, m->inv64, nval * sizeof(double));
    if(inv32) memcpy(inv32, m->inv32, nval * sizeof(float));
    return m->nblk;
}

/* MASPreconditioner::preconditioning (SG/MASPreconditioner.cu:2210-2251):
 * BuildMultiLevelR (:727-845), SchwarzLocalXSym_block3 -> _schwarzLocalXSym6
 * (:954-1024, :2125-2137), CollectFinalZ (:848-877). */
int or_mas_apply(or_mas* m, const double* r, double* z)
{
    const int b = m->bank, L = m->levelnum, N = m->N, Mm = m->Mm, T = m->total;
    if(!m->hess)
        return -1;
    const int dbl = (m->precision == 2);
    double* R64 = (double*)xcalloc((size_t)T * 3, sizeof(double));
    double* Z64 = (double*)xcalloc((size_t)T * 3, sizeof(double));
    float*  R32 = (float*)xcalloc((size_t)T * 3, sizeof(float));
    float*  Z32 = (float*)xcalloc((size_t)T * 3, sizeof(float));
    /* level 0 */
    for(int s = 0; s < Mm; s++)
    {
        int idx = m->part_map[s];
        for(int d = 0; d < 3; d++)
        {
            double v        = idx >= 0 ? r[3 * (size_t)idx + d] : 0.0;
            R64[3 * s + d]  = v;
            R32[3 * s + d]  = (float)v;
        }
    }
    /* component sums pushed up the chain */
    for(int h = 0; h < Mm / b; h++)
        for(int lane = 0; lane < b; lane++)
        {
            int idx = m->part_map[h * b + lane];
            if(idx < 0)
                continue;
            unsigned msk = m->fine_mask[idx];
            if(popc(msk & lanemask_lt(lane)) != 0)
                continue; /* not the component leader */
            double s64[3] = {0, 0, 0};
            float  s32[3] = {0, 0, 0};
            for(int j = 0; j < b; j++)
                if(msk & (1u << j))
                    for(int d = 0; d < 3; d++)
                    {
                        s64[d] += R64[3 * (h * b + j) + d];
                        s32[d] += R32[3 * (h * b + j) + d];
                    }
            if(L > 1)
            {
                int nx = m->going_next[idx];
                for(int d = 0; d < 3; d++)
                {
                    R64[3 * (size_t)nx + d] = s64[d];
                    R32[3 * (size_t)nx + d] = s32[d];
                }
            }
        }
    /* levels >= 2: each coarse node sums its children, which all lie in one
     * bank of the level below, lanes ascending (the reference pushes every
     * component up the whole chain with atomics; same sums, defined order) */
    for(int lvl = 2; lvl < L; lvl++)
    {
        const int beg = m->level_size[2 * (lvl - 1) + 1], cnt = m->level_size[2 * (lvl - 1)];
        for(int k = 0; k * b < cnt; k++)
            for(int lane = 0; lane < b && k * b + lane < cnt; lane++)
            {
                const int node = beg + k * b + lane;
                const int par  = m->going_next[node];
                int lead       = 1;
                for(int j = 0; j < lane; j++)
                    if(m->going_next[beg + k * b + j] == par)
                        lead = 0;
                if(!lead)
                    continue;
                double s64[3] = {0, 0, 0};
                float  s32[3] = {0, 0, 0};
                for(int j = lane; j < b && k * b + j < cnt; j++)
                    if(m->going_next[beg + k * b + j] == par)
                        for(int d = 0; d < 3; d++)
                        {
                            s64[d] += R64[3 * (size_t)(beg + k * b + j) + d];
                            s32[d] += R32[3 * (size_t)(beg + k * b + j) + d];
                        }
                for(int d = 0; d < 3; d++)
                {
                    R64[3 * (size_t)par + d] = s64[d];
                    R32[3 * (size_t)par + d] = s32[d];
                }
            }
    }
    /* Schwarz: per bank z = P r, columns ascending, fma chains */
    const size_t bsym = (size_t)m->bsym;
    if(is_factored(m->precision))
    {
        /* factored tiles: y = W r (J <= I), z = W^T y (J >= I), J ascending
           within each part; with M = b / 2, pass 1 sums a row I >= M as
           (J < M) + (M <= J <= I) and pass 2 a row I < M as (I <= J < M) +
           (J >= M), each part its own chain from 0, the two added last (the
           library's lane-balanced order) */
        const int M = b / 2;
#pragma omp parallel for schedule(static)
        for(int B = 0; B < T / b; B++)
        {
            float y[32][3];
            for(int rl = 0; rl < b; rl++)
            {
                float a[3] = {0, 0, 0}, h[3] = {0, 0, 0};
                for(int cl = 0; cl <= rl; cl++)
                {
                    const float* P = m->inv32 + ((size_t)B * bsym + sym_index(b, cl, rl)) * 9;
                    const float* x = R32 + 3 * (size_t)(B * b + cl);
                    float* acc = (rl >= M && cl >= M) ? h : a;
                    for(int d = 0; d < 3; d++)
                        for(int k = 0; k < 3; k++)
                            acc[d] = fmaf(P[d + 3 * k], x[k], acc[d]);
                }
                for(int d = 0; d < 3; d++)
                    y[rl][d] = rl >= M ? a[d] + h[d] : a[d];
            }
            for(int rl = 0; rl < b; rl++)
            {
                float a[3] = {0, 0, 0}, l[3] = {0, 0, 0};
                for(int cl = rl; cl < b; cl++)
                {
                    const float* P = m->inv32 + ((size_t)B * bsym + sym_index(b, rl, cl)) * 9;
                    float* acc = (rl < M && cl < M) ? l : a;
                    for(int d = 0; d < 3; d++)
                        for(int k = 0; k < 3; k++)
                            acc[d] = fmaf(P[k + 3 * d], y[cl][k], acc[d]);
                }
                for(int d = 0; d < 3; d++)
                    Z32[3 * ((size_t)B * b + rl) + d] = rl < M ? l[d] + a[d] : a[d];
            }
        }
    }
    else
#pragma omp parallel for schedule(static)
    for(int B = 0; B < T / b; B++)
        for(int rl = 0; rl < b; rl++)
        {
            double a64[3] = {0, 0, 0};
            float  a32[3] = {0, 0, 0};
            for(int cl = 0; cl < b; cl++)
            {
                size_t base;
                int tr;
                if(cl >= rl) { base = ((size_t)B * bsym + sym_index(b, rl, cl)) * 9; tr = 0; }
                else { base = ((size_t)B * bsym + sym_index(b, cl, rl)) * 9; tr = 1; }
                const int node = B * b + cl;
                for(int a = 0; a < 3; a++)
                    for(int c = 0; c < 3; c++)
                    {
                        size_t e = tr ? base + c + 3 * a : base + a + 3 * c;
                        if(dbl)
                            a64[a] = fma(m->inv64[e], R64[3 * (size_t)node + c], a64[a]);
                        else
                            a32[a] = fmaf(m->inv32[e], R32[3 * (size_t)node + c], a32[a]);
                    }
            }
            for(int a = 0; a < 3; a++)
            {
                Z64[3 * ((size_t)B * b + rl) + a] = a64[a];
                Z32[3 * ((size_t)B * b + rl) + a] = a32[a];
            }
        }
    /* __collectFinalZ_new */
#pragma omp parallel for schedule(static)
    for(int v = 0; v < N; v++)
    {
        int rd = m->real_map[v];
        if(dbl)
        {
            double c[3] = {Z64[3 * rd], Z64[3 * rd + 1], Z64[3 * rd + 2]};
            for(int i = 1; i < L; i++)
            {
                int now = m->coarse_table[6 * (size_t)v + i - 1];
                for(int d = 0; d < 3; d++)
                    c[d] += Z64[3 * (size_t)now + d];
            }
            for(int d = 0; d < 3; d++)
                z[3 * (size_t)v + d] = c[d];
        }
        else
        {
            float c[3] = {Z32[3 * rd], Z32[3 * rd + 1], Z32[3 * rd + 2]};
            for(int i = 1; i < L; i++)
            {
                int now = m->coarse_table[6 * (size_t)v + i - 1];
                for(int d = 0; d < 3; d++)
                    c[d] += Z32[3 * (size_t)now + d];
            }
            for(int d = 0; d < 3; d++)
                z[3 * (size_t)v + d] = (double)c[d];
        }
    }
    free(R64); free(Z64); free(R32); free(Z32);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* PCG (SG/linear_system/solver/pcg_solver.cu:155-304) with the reference's  */
/* preconditioner order (global_linear_system.cu:509-522): the global one    */
/* (3x3 block-Jacobi, DiagPreconditioner diag_preconditioner.cu:9-66) or an  */
/* identity copy, then the ABD 12x12 block-Jacobi                            */
/* (setup_abd_system_gradient_and_hessian.cu:603-645), then the MAS on the   */
/* FEM sub-range.                                                            */
/* ------------------------------------------------------------------------ */
static int invert_dense(double* A, int n)
{
    /* LU with partial pivoting, in place -> inverse (Gauss-Jordan form) */
    int* piv = (int*)malloc(sizeof(int) * (size_t)n);
    for(int i = 0; i < n; i++) piv[i] = i;
    for(int k = 0; k < n; k++)
    {
        int p = k;
        double best = fabs(A[k * n + k]);
        for(int i = k + 1; i < n; i++)
            if(fabs(A[i * n + k]) > best) { best = fabs(A[i * n + k]); p = i; }
        if(best == 0) { free(piv); return -1; }
        if(p != k)
        {
            for(int j = 0; j < n; j++) { double t = A[k * n + j]; A[k * n + j] = A[p * n + j]; A[p * n + j] = t; }
            int t = piv[k]; piv[k] = piv[p]; piv[p] = t;
        }
        double d = A[k * n + k];
        A[k * n + k] = 1.0;
        for(int j = 0; j < n; j++) A[k * n + j] /= d;
        for(int i = 0; i < n; i++)
        {
            if(i == k) continue;
            double f = A[i * n + k];
            A[i * n + k] = 0.0;
            for(int j = 0; j < n; j++) A[i * n + j] -= f * A[k * n + j];
        }
    }
    /* undo the column permutation implied by the row swaps */
    double* T = (double*)malloc(sizeof(double) * (size_t)n * n);
    for(int i = 0; i < n; i++)
        for(int j = 0; j < n; j++)
            T[i * n + piv[j]] = A[i * n + j];
    memcpy(A, T, sizeof(double) * (size_t)n * n);
    free(T);
    free(piv);
    return 0;
}

typedef struct
{
    int nrows;
    int64_t* ptr; /* full CSR of 3x3 blocks (both triangles) */
    int* col;
    double* val;  /* row-major 3x3 */
} or_csr;

static void csr_build(or_csr* A, const double* vals, const int* rows, const int* cols, int nb, int nrows)
{
    A->nrows = nrows;
    A->ptr   = (int64_t*)xcalloc((size_t)nrows + 1, sizeof(int64_t));
    for(int k = 0; k < nb; k++)
    {
        A->ptr[rows[k] + 1]++;
        if(rows[k] != cols[k]) A->ptr[cols[k] + 1]++;
    }
    for(int i = 0; i < nrows; i++) A->ptr[i + 1] += A->ptr[i];
    int64_t nnz = A->ptr[nrows];
    A->col = (int*)xcalloc((size_t)nnz, sizeof(int));
    A->val = (double*)xcalloc((size_t)nnz * 9, sizeof(double));
    int64_t* fill = (int64_t*)xcalloc((size_t)nrows, sizeof(int64_t));
    for(int k = 0; k < nb; k++)
    {
        int i = rows[k], j = cols[k];
        const double* H = vals + 9 * (size_t)k;
        int64_t p = A->ptr[i] + fill[i]++;
        A->col[p] = j;
        for(int a = 0; a < 3; a++)
            for(int c = 0; c < 3; c++) A->val[9 * p + 3 * a + c] = H[a + 3 * c];
        if(i != j)
        {
            p = A->ptr[j] + fill[j]++;
            A->col[p] = i;
            for(int a = 0; a < 3; a++)
                for(int c = 0; c < 3; c++) A->val[9 * p + 3 * a + c] = H[c + 3 * a];
        }
    }
    free(fill);
}
static void csr_free(or_csr* A) { free(A->ptr); free(A->col); free(A->val); }

static void csr_spmv(const or_csr* A, const double* x, double* y)
{
#pragma omp parallel for schedule(static)
    for(int i = 0; i < A->nrows; i++)
    {
        double s0 = 0, s1 = 0, s2 = 0;
        for(int64_t p = A->ptr[i]; p < A->ptr[i + 1]; p++)
        {
            const double* H = A->val + 9 * p;
            const double* v = x + 3 * (size_t)A->col[p];
            s0 += H[0] * v[0] + H[1] * v[1] + H[2] * v[2];
            s1 += H[3] * v[0] + H[4] * v[1] + H[5] * v[2];
            s2 += H[6] * v[0] + H[7] * v[1] + H[8] * v[2];
        }
        y[3 * (size_t)i] = s0; y[3 * (size_t)i + 1] = s1; y[3 * (size_t)i + 2] = s2;
    }
}
static double pdot(const double* a, const double* b, int n)
{
    double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for(int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

int or_pcg(const double* vals, const int* rows, const int* cols, int nb, int nrows,
           const double* b, double* x, const or_pcg_cfg* cfg, or_mas* mas, or_pcg_report* rep)
{
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
#ifdef _OPENMP
    int saved = omp_get_max_threads();
    if(cfg->nthreads > 0) omp_set_num_threads(cfg->nthreads);
#endif
    const int n = 3 * nrows;
    or_csr A;
    csr_build(&A, vals, rows, cols, nb, nrows);
    /* preconditioner assembly */
    double* D = NULL;
    if(cfg->precond == 1)
    {
        D = (double*)xcalloc((size_t)nrows * 9, sizeof(double));
        for(int k = 0; k < nb; k++)
            if(rows[k] == cols[k])
            {
                double M[9];
                for(int a = 0; a < 3; a++)
                    for(int c = 0; c < 3; c++) M[3 * a + c] = vals[9 * (size_t)k + a + 3 * c];
                invert_dense(M, 3);
                memcpy(D + 9 * (size_t)rows[k], M, sizeof(M));
            }
    }
    double* P12 = NULL;
    if(cfg->abd_bodies > 0)
    {
        P12 = (double*)xcalloc((size_t)cfg->abd_bodies * 144, sizeof(double));
        for(int k = 0; k < nb; k++)
        {
            int i = rows[k], j = cols[k];
            if(i / 4 != j / 4 || i >= 4 * cfg->abd_bodies) continue;
            double* P = P12 + 144 * (size_t)(i / 4);
            const double* H = vals + 9 * (size_t)k;
            for(int a = 0; a < 3; a++)
                for(int c = 0; c < 3; c++)
                {
                    P[((i % 4) * 3 + a) * 12 + (j % 4) * 3 + c] = H[a + 3 * c];
                    if(i != j) P[((j % 4) * 3 + c) * 12 + (i % 4) * 3 + a] = H[a + 3 * c];
                }
        }
        for(int q = 0; q < cfg->abd_bodies; q++) invert_dense(P12 + 144 * (size_t)q, 12);
    }
    double *r = (double*)xcalloc((size_t)n, 8), *z = (double*)xcalloc((size_t)n, 8),
           *p = (double*)xcalloc((size_t)n, 8), *Ap = (double*)xcalloc((size_t)n, 8);
#define OR_APPLY()                                                                         \
    do {                                                                                   \
        if(cfg->precond == 1) {                                                            \
            _Pragma("omp parallel for schedule(static)")                                   \
            for(int i = 0; i < nrows; i++) {                                               \
                const double* M = D + 9 * (size_t)i;                                       \
                const double* v = r + 3 * (size_t)i;                                       \
                for(int a = 0; a < 3; a++)                                                 \
                    z[3 * (size_t)i + a] = M[3 * a] * v[0] + M[3 * a + 1] * v[1] + M[3 * a + 2] * v[2]; \
            }                                                                              \
        } else memcpy(z, r, sizeof(double) * (size_t)n);                                  \
        for(int q = 0; q < cfg->abd_bodies; q++) {                                         \
            const double* M = P12 + 144 * (size_t)q;                                       \
            for(int a = 0; a < 12; a++) {                                                  \
                double s = 0;                                                              \
                for(int c = 0; c < 12; c++) s += M[a * 12 + c] * r[12 * (size_t)q + c];    \
                z[12 * (size_t)q + a] = s;                                                 \
            }                                                                              \
        }                                                                                  \
        if(cfg->precond == 2 && mas)                                                       \
            or_mas_apply(mas, r + 3 * (size_t)cfg->fem_offset, z + 3 * (size_t)cfg->fem_offset); \
    } while(0)

    int max_iter = cfg->max_iter == 0 ? n : cfg->max_iter;
    /* start guess: x0 scaled by the A-norm-optimal alpha = x0.b / x0.A x0
       (0 unless positive), rejected when ||b - alpha A x0|| > ||b||; the
       convergence test is then relative to ||b|| */
    double bb = 0;
    int warm = cfg->initial_guess;
    rep->x0_scale = 0;
    rep->x0_rejected = 0;
    if(warm)
    {
        csr_spmv(&A, x, Ap);
        const double xax = pdot(x, Ap, n), xb = pdot(x, b, n);
        bb = pdot(b, b, n);
        const double alpha = (xax > 0 && xb > 0) ? xb / xax : 0.0;
        for(int i = 0; i < n; i++) { r[i] = b[i] - alpha * Ap[i]; x[i] = alpha * x[i]; }
        const double rr = pdot(r, r, n);
        rep->x0_scale = alpha;
        rep->x0_rejected = !(rr <= bb) || alpha == 0.0;
    }
    if(!warm || rep->x0_rejected)
    {
        for(int i = 0; i < n; i++) x[i] = 0;
        memcpy(r, b, sizeof(double) * (size_t)n);
    }
    OR_APPLY();
    double rz = pdot(r, z, n);
    memcpy(p, z, sizeof(double) * (size_t)n);
    double rz0 = rz, rr0 = 0;
    if(!cfg->use_preconditioned_norm) rr0 = warm ? bb : pdot(r, r, n);
    const double rel2 = cfg->rel_tol * cfg->rel_tol, abs2 = cfg->abs_tol * cfg->abs_tol;
    int k;
    for(k = 1; k < max_iter; ++k)
    {
        csr_spmv(&A, p, Ap);
        double alpha = rz / pdot(p, Ap, n);
#pragma omp parallel for schedule(static)
        for(int i = 0; i < n; i++) { x[i] = x[i] + alpha * p[i]; r[i] = r[i] - alpha * Ap[i]; }
        if(k % 10 == 0)
        {
            csr_spmv(&A, x, Ap);
#pragma omp parallel for schedule(static)
            for(int i = 0; i < n; i++) r[i] = b[i] - Ap[i];
        }
        OR_APPLY();
        double rz_new = pdot(r, z, n);
        if(k % 10 == 0)
        {
            if(cfg->use_preconditioned_norm)
            {
                if(rz_new <= rel2 * rz0 || rz_new <= abs2) break;
            }
            else
            {
                double rr = pdot(r, r, n);
                if(rr <= rel2 * rr0 || rr <= abs2) break;
            }
        }
        double beta = rz_new / rz;
#pragma omp parallel for schedule(static)
        for(int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        rz = rz_new;
    }
#undef OR_APPLY
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if(rep)
    {
        csr_spmv(&A, x, Ap);
        double rr = 0, bb = 0;
        for(int i = 0; i < n; i++) { double d = b[i] - Ap[i]; rr += d * d; bb += b[i] * b[i]; }
        rep->iterations   = k;
        rep->rel_residual = bb > 0 ? sqrt(rr / bb) : sqrt(rr);
        rep->rz0          = rz0;
        rep->rr0          = rr0;
        rep->ms           = (t1.tv_sec - t0.tv_sec) * 1e3 + (t1.tv_nsec - t0.tv_nsec) * 1e-6;
    }
    free(r); free(z); free(p); free(Ap); free(D); free(P12);
    csr_free(&A);
#ifdef _OPENMP
    omp_set_num_threads(saved);
#endif
    return k;
}
