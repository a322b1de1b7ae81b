// grid.cuh — blocked layout of the background grid.
//
// The G^3 grid is stored as NB^3 blocks of 4x4x4 nodes (NB = ceil(G/4)),
// each block 64 consecutive float4 = 1 KiB: block (bi, bj, bk) at
// ((bi*NB + bj)*NB + bk), node (i&3, j&3, k&3) inside it at
// ((i&3)<<4 | (j&3)<<2 | (k&3)). A 4^3 block is the unit of the sparse grid
// update (one flag byte per block) and is contiguous in HBM, so a block is
// read or written with fully coalesced 16-byte accesses.
#pragma once
#include "mat3.cuh"

namespace empm {

EMPM_HD int grid_nb(int G) { return (G + 3) >> 2; }

EMPM_HD long long grid_nodes_padded(int G) {
    const long long nb = grid_nb(G);
    return nb * nb * nb * 64;
}

EMPM_HD int block_of(int i, int j, int k, int NB) { return ((i >> 2) * NB + (j >> 2)) * NB + (k >> 2); }

EMPM_HD long long node_addr(int i, int j, int k, int NB) {
    return ((long long)block_of(i, j, k, NB) << 6) | ((i & 3) << 4) | ((j & 3) << 2) | (k & 3);
}

// inverse of node_addr for a node inside block b
EMPM_HD void node_coords(long long addr, int NB, int& i, int& j, int& k) {
    const long long b = addr >> 6;
    const int o = (int)(addr & 63);
    const int bk = (int)(b % NB);
    const int bj = (int)((b / NB) % NB);
    const int bi = (int)(b / ((long long)NB * NB));
    i = (bi << 2) | (o >> 4);
    j = (bj << 2) | ((o >> 2) & 3);
    k = (bk << 2) | (o & 3);
}

}  // namespace empm
