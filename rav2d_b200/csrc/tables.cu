// The AV2 constant tables in device global memory, one copy per device,
// generated from the reference sources (see gen_av2_tables.py).
#include "r2g_common.cuh"

#define R2G_TABLE(type, name) __device__ const type d_##name
#include "av2_tables.h"
#undef R2G_TABLE

#define SYM(name, field)                                                         \
    do {                                                                         \
        void *p = nullptr;                                                       \
        cudaError_t e = cudaGetSymbolAddress(&p, d_##name);                      \
        if (e != cudaSuccess) return e;                                          \
        t->field = reinterpret_cast<decltype(t->field)>(p);                      \
    } while (0)

cudaError_t r2g_get_tables(DevTables *t) {
    SYM(CDEF_DIRECTIONS, CDEF_DIRECTIONS);
    SYM(CCSO_QUANT_SZ, CCSO_QUANT_SZ);
    SYM(CCSO_OFFSET, CCSO_OFFSET);
    SYM(DEBLOCK_SIDE_THRESHOLDS, DEBLOCK_SIDE_THRESHOLDS);
    SYM(PC_WIENER_FILTERS, PC_WIENER_FILTERS);
    SYM(PC_WIENER_SUB_CLASSIFY, PC_WIENER_SUB_CLASSIFY);
    SYM(PC_WIENER_SUB_CLASSIFY_NS, PC_WIENER_SUB_CLASSIFY_NS);
    SYM(GAUSSIAN_SEQUENCE, GAUSSIAN_SEQUENCE);
    SYM(PC_WIENER_LUT_TO_CLASS, PC_WIENER_LUT_TO_CLASS);
    SYM(GDF_ALPHA, GDF_ALPHA);
    SYM(GDF_WEIGHT, GDF_WEIGHT);
    SYM(GDF_BIAS, GDF_BIAS);
    SYM(GDF_INTRA_ERROR, GDF_INTRA_ERROR);
    SYM(GDF_INTER_ERROR, GDF_INTER_ERROR);
    SYM(BLOCK_DIMENSIONS, BLOCK_DIMENSIONS);
    SYM(TXFM_DIMENSIONS, TXFM_DIMENSIONS);
    SYM(MAX_TXFM_SIZE_FOR_BS, MAX_TXFM_SIZE_FOR_BS);
    SYM(TX_PART_TBL, TX_PART_TBL);
    return cudaSuccess;
}
