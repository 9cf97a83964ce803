// nan_pairwise.h -- numpy's float64 summation of a float32 array, fed one
// term at a time (the support estimate of nan_wse.cu sums its terms this way
// to equal the reference's Python form bit for bit). Plain C++ as well as
// CUDA device code, so the host test suite compiles the same struct and
// checks it against numpy.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define NAN_PAIRWISE_FN __host__ __device__
#else
#define NAN_PAIRWISE_FN
#endif

namespace nan_pairwise {

constexpr uint32_t kBuffer = 8192;  // numpy's default ufunc buffer (elements)

// For a term count known before the first term: buffers of 8192 terms whose
// sums are added in order; each buffer by the pairwise scheme -- above 128
// terms the left part takes n/2 rounded down to a multiple of 8; a leaf of 8
// to 128 terms keeps eight running sums over its whole 8-blocks, combines
// them pairwise and adds the remainder in order; a leaf of fewer than 8 terms
// is summed in order from 0. The path from a buffer's root to the current
// leaf is a stack of (node length, left sum, taking the right child); a
// buffer of 8192 terms is at most 7 levels deep.
struct Feed {
    double acc[8];
    double leaf, total;
    double frame_left[8];
    uint32_t frame_len[8];
    uint32_t remaining, leaf_len, leaf_pos, depth, right;

    NAN_PAIRWISE_FN void descend(uint32_t len) {
        while (len > 128u) {
            frame_len[depth] = len;
            right &= ~(1u << depth);
            ++depth;
            len = len / 2u - (len / 2u) % 8u;
        }
        leaf_len = len;
        leaf_pos = 0;
        leaf = 0.0;
    }
    NAN_PAIRWISE_FN void next_buffer() {
        const uint32_t len = remaining < kBuffer ? remaining : kBuffer;
        remaining -= len;
        depth = 0;
        right = 0;
        descend(len);
    }
    NAN_PAIRWISE_FN void begin(uint32_t n) {
        total = 0.0;
        remaining = n;
        if (n) next_buffer();
    }
    NAN_PAIRWISE_FN void finish_leaf() {
        double v = leaf;
        for (;;) {
            if (depth == 0) {
                total = total + v;
                if (remaining) next_buffer();
                return;
            }
            const uint32_t d = depth - 1;
            if (!((right >> d) & 1u)) {  // the left child is done: take the right one
                frame_left[d] = v;
                right |= 1u << d;
                descend(frame_len[d] - (frame_len[d] / 2u - (frame_len[d] / 2u) % 8u));
                return;
            }
            v = frame_left[d] + v;
            depth = d;
        }
    }
    NAN_PAIRWISE_FN void push(double v) {
        if (leaf_len < 8u) {
            leaf += v;
        } else {
            const uint32_t blocks_end = leaf_len - leaf_len % 8u;
            if (leaf_pos < blocks_end) {
                const uint32_t j = leaf_pos & 7u;
                acc[j] = leaf_pos < 8u ? v : acc[j] + v;
                if (leaf_pos + 1u == blocks_end)
                    leaf = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
            } else {
                leaf += v;
            }
        }
        if (++leaf_pos == leaf_len) finish_leaf();
    }
};

}  // namespace nan_pairwise
