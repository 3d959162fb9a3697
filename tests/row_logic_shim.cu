// Host entry points over two device functions of the row stage, for the CPU
// tests (tests/test_row_logic.py): walk_row (the winding walk of one AA row
// into spans) and sweep_cells (four AA rows' spans into a pixel row's
// coverage cells). Both are __host__ __device__; the kernels run the same
// source on the GPU.
#include <cstdint>

#include "../pdf-raster_b200/csrc/rrb_kernels.cuh"

namespace {

struct RowIn {
    const int32_t *x0s, *x1s, *counts;
    __host__ __device__ void operator()(int i, int32_t& a, int32_t& b, int32_t& c) const {
        a = x0s[i];
        b = x1s[i];
        c = counts[i];
    }
};

struct SpanOut {
    int32_t *x0, *x1;
    __host__ __device__ void operator()(int k, int32_t a, int32_t b) const {
        x0[k] = a;
        x1[k] = b;
    }
};

struct Bounds {
    const int32_t *x0, *x1;
    int stride;
    __host__ __device__ int32_t operator()(int k, int i, bool end) const {
        return end ? x1[k * stride + i] : x0[k * stride + i];
    }
};

struct CellOut {
    uint32_t* cells;
    __host__ __device__ void operator()(int q, uint32_t c) const { cells[q] = c; }
};

}  // namespace

extern "C" int rl_walk_row(const int32_t* x0s, const int32_t* x1s, const int32_t* counts, int n, int eo,
                           int32_t aa_width, int32_t lo, int32_t hi, int32_t* span_x0, int32_t* span_x1,
                           uint32_t* nonterminating) {
    uint32_t nt = 0;
    const int ns = rrb::walk_row(n, eo ? 1 : ~0, aa_width, lo, hi, RowIn{x0s, x1s, counts}, SpanOut{span_x0, span_x1},
                                 nt);
    *nonterminating = nt;
    return ns;
}

// n4[k] spans of sub-row k at span_x0/x1[k * stride + i]; cells[] receives
// x0 | (len - 1) << 14 | (cov - 1) << 28 per cell, at most 4 * (n4 sum).
extern "C" int rl_sweep_cells(const int32_t* n4, const int32_t* span_x0, const int32_t* span_x1, int stride,
                              uint32_t* cells) {
    const int n[4] = {n4[0], n4[1], n4[2], n4[3]};
    return rrb::sweep_cells(n, Bounds{span_x0, span_x1, stride}, CellOut{cells});
}
