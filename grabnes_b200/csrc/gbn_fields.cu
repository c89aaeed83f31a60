// Sparse-product kernels of the field-batched layout: one field-free matrix serves right-hand sides of
// many perpendicular fields.  Each stored entry holds the field-free hopping and its Peierls phase per
// flux quantum (HamPeierlsPeriodicGauge, lanczosKuboCode/Src/ham.F90:12834-12882, is linear in the
// number of flux quanta m), and the threads of a right-hand side of m quanta rotate the entry by
// exp(2 pi i frac(m tau)) as they use it.  One matrix stream then feeds every field of a tile instead
// of one assembled matrix per field.  The tile-table kernels read the same records with the rotations
// done once per tile (build_field_table): complex values per thread slot.
#include "gbn_step.cuh"

namespace gbn {

template <typename VT, int G>
static StepFn pick_field_g(int rpt, int tpr, bool staged)
{
#define GBN_CASE(RP, TP) \
    if (rpt == RP && tpr == TP) return staged ? k_spmm_staged<VT, false, G, RP, TP, true> : k_spmm_step<VT, false, G, RP, TP, true>;
    GBN_CASE(1, 1) GBN_CASE(1, 2) GBN_CASE(1, 4) GBN_CASE(1, 8) GBN_CASE(1, 16) GBN_CASE(1, 32)
    GBN_CASE(2, 1) GBN_CASE(2, 2) GBN_CASE(2, 4) GBN_CASE(2, 8) GBN_CASE(2, 16)
    if constexpr (sizeof(VT) == 4) {
        GBN_CASE(4, 1) GBN_CASE(4, 2) GBN_CASE(4, 4) GBN_CASE(4, 8)
    }
#undef GBN_CASE
    return nullptr;
}

template <typename VT, int G>
static StepFn pick_table_g(int rpt, int tpr, bool staged)
{
#define GBN_CASE(RP, TP)                                                                                        \
    if (rpt == RP && tpr == TP)                                                                                 \
        return staged ? k_spmm_staged<VT, true, G, RP, TP, false, kColUnroll, true, 1, true>                     \
                      : k_spmm_step<VT, true, G, RP, TP, false, kColUnroll, true>;
    GBN_CASE(1, 1) GBN_CASE(1, 2) GBN_CASE(1, 4) GBN_CASE(1, 8) GBN_CASE(1, 16) GBN_CASE(1, 32)
    GBN_CASE(2, 1) GBN_CASE(2, 2) GBN_CASE(2, 4) GBN_CASE(2, 8) GBN_CASE(2, 16)
    if constexpr (sizeof(VT) == 4) {
        GBN_CASE(4, 1) GBN_CASE(4, 2) GBN_CASE(4, 4) GBN_CASE(4, 8)
    }
#undef GBN_CASE
    return nullptr;
}

StepFn field_table_kernel(int prec, int G, int rpt, int tpr, bool staged)
{
    if (prec == GBN_MIXED) {
        if (G == 1) return pick_table_g<float, 1>(rpt, tpr, staged);
        if (G == 2) return pick_table_g<float, 2>(rpt, tpr, staged);
        if (G == 4) return pick_table_g<float, 4>(rpt, tpr, staged);
    } else {
        if (G == 1) return pick_table_g<double, 1>(rpt, tpr, staged);
        if (G == 2) return pick_table_g<double, 2>(rpt, tpr, staged);
        if (G == 4) return pick_table_g<double, 4>(rpt, tpr, staged);
    }
    return nullptr;
}

// the fused field product at the widest loads (mixed precision 4 right-hand sides per thread, FP64 2):
// registers for one block per SM, or bounded for two (min_blocks 2)
template <typename VT, int G, int MINB>
static StepFn pick_field_fused_g(int tpr)
{
    constexpr int RP = sizeof(VT) == 4 ? 4 : 2;
    if (tpr == 2) return k_spmm_staged<VT, false, G, RP, 2, true, kColUnroll, true, MINB, false, true>;
    if (tpr == 4) return k_spmm_staged<VT, false, G, RP, 4, true, kColUnroll, true, MINB, false, true>;
    if (tpr == 8) return k_spmm_staged<VT, false, G, RP, 8, true, kColUnroll, true, MINB, false, true>;
    if constexpr (sizeof(VT) == 8) {
        if (tpr == 16) return k_spmm_staged<VT, false, G, RP, 16, true, kColUnroll, true, MINB, false, true>;
    }
    return nullptr;
}

// one right-hand side per thread: a sweep of one vector per field (the drop-in driver's DOS sweeps)
template <typename VT, int G, int MINB>
static StepFn pick_field_fused_single(int tpr)
{
    if (tpr == 8) return k_spmm_staged<VT, false, G, 1, 8, true, kColUnroll, true, MINB, false, true>;
    if (tpr == 16) return k_spmm_staged<VT, false, G, 1, 16, true, kColUnroll, true, MINB, false, true>;
    if (tpr == 32) return k_spmm_staged<VT, false, G, 1, 32, true, kColUnroll, true, MINB, false, true>;
    return nullptr;
}

template <typename VT>
static StepFn pick_field_fused(int G, int rpt, int tpr, int min_blocks)
{
    if (rpt == 1) {
        if (G == 1) return min_blocks == 2 ? pick_field_fused_single<VT, 1, 2>(tpr) : pick_field_fused_single<VT, 1, 1>(tpr);
        if (G == 2) return min_blocks == 2 ? pick_field_fused_single<VT, 2, 2>(tpr) : pick_field_fused_single<VT, 2, 1>(tpr);
        return nullptr;
    }
    if (rpt != (sizeof(VT) == 4 ? 4 : 2)) return nullptr;
    if (min_blocks == 2) {
        if (G == 1) return pick_field_fused_g<VT, 1, 2>(tpr);
        if (G == 2) return pick_field_fused_g<VT, 2, 2>(tpr);
        return nullptr;
    }
    if (G == 1) return pick_field_fused_g<VT, 1, 1>(tpr);
    if (G == 2) return pick_field_fused_g<VT, 2, 1>(tpr);
    if constexpr (sizeof(VT) == 4) {
        if (G == 4) return pick_field_fused_g<VT, 4, 1>(tpr);
    }
    return nullptr;
}

StepFn field_fused_kernel(int prec, int G, int rpt, int tpr, int min_blocks)
{
    if (prec == GBN_MIXED) return pick_field_fused<float>(G, rpt, tpr, min_blocks);
    return pick_field_fused<double>(G, rpt, tpr, min_blocks);
}

StepFn field_step_kernel(int prec, int G, int rpt, int tpr, bool staged)
{
    if (prec == GBN_MIXED) {
        if (G == 1) return pick_field_g<float, 1>(rpt, tpr, staged);
        if (G == 2) return pick_field_g<float, 2>(rpt, tpr, staged);
        if (G == 4) return pick_field_g<float, 4>(rpt, tpr, staged);
    } else {
        if (G == 1) return pick_field_g<double, 1>(rpt, tpr, staged);
        if (G == 2) return pick_field_g<double, 2>(rpt, tpr, staged);
        if (G == 4) return pick_field_g<double, 4>(rpt, tpr, staged);
    }
    return nullptr;
}

}  // namespace gbn
