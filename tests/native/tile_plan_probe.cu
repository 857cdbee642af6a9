// Host-only probe of the SpMV setup in rowblock.cuh (tile plan, long-row
// chunks, row-start bitmap, padding, tile-kernel choice), for the CPU tests.
// Reads "nrow nnz" then nrow+1 row starts and nnz column indices on stdin;
// prints the plan as JSON.  Calls no CUDA API.
#include "rowblock.cuh"

#include <cstdio>
#include <vector>

int main()
{
    int nrow = 0, nnz = 0;
    if (scanf("%d %d", &nrow, &nnz) != 2 || nrow < 0 || nnz < 0) return 2;
    std::vector<int> rp(nrow + 1), ci(nnz);
    for (int &v : rp)
        if (scanf("%d", &v) != 1) return 2;
    for (int &v : ci)
        if (scanf("%d", &v) != 1) return 2;
    hpr::TilePlan plan;
    hpr::build_tile_plan(rp, plan);
    std::vector<unsigned char> heads;
    hpr::build_heads(rp, heads);
    printf("{\"padded_nnz\": %zu, \"staged\": %d, \"tiles\": [", hpr::padded_nnz((size_t)nnz),
           hpr::choose_staged(rp, ci));
    for (size_t i = 0; i < plan.tiles.size(); ++i)
        printf("%s[%d, %d, %d, %d]", i ? ", " : "", plan.tiles[i].x, plan.tiles[i].y, plan.tiles[i].z,
               plan.tiles[i].w);
    printf("], \"chunks\": [");
    for (size_t i = 0; i < plan.chunks.size(); ++i)
        printf("%s[%d, %d, %d, %d]", i ? ", " : "", plan.chunks[i].x, plan.chunks[i].y, plan.chunks[i].z,
               plan.chunks[i].w);
    printf("], \"long_rows\": [");
    for (size_t i = 0; i < plan.long_rows.size(); ++i)
        printf("%s[%d, %d]", i ? ", " : "", plan.long_rows[i].x, plan.long_rows[i].y);
    printf("], \"heads\": [");
    for (size_t i = 0; i < heads.size(); ++i) printf("%s%u", i ? ", " : "", (unsigned)heads[i]);
    printf("]}\n");
    return 0;
}
