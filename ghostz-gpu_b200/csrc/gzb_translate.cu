// gzb_translate.cu -- six-frame translation of DNA reads into translated
// queries, on the device (query preparation of `aln -q d -t p`).
//
// The layout is the reference's TranslatedDnaQuery
// (src/translated_dna_query.cpp:44-74): a leading delimiter, then per frame
// (forward offsets 0, 1, 2, then offsets 0, 1, 2 of the reverse
// complementary strand) its codons as protein codes, one extra delimiter
// when the frame has fewer than length/3 codons, and a closing delimiter;
// 7 + 6 * (length / 3) codes in all.  Codons follow Translator::Translate
// (src/translator.cpp:104-142): the codon table is matched case-sensitively
// on the strand's letters, its "stopped" flag is never set, so every codon
// in the table translates and every other one becomes the unknown letter X.
// The reverse strand is built by DnaSequence::GetComplementaryStrand
// (src/dna_sequence.h:28-42): A/a->T, C/c->G, G/g->C, T/t->A, else N.
//
// One warp per read: lane j translates codon j of all six frames, so for
// each frame the stores of a warp are contiguous; the read's bases come
// from L1 (a lane reads five consecutive bases per strand).
#include <cuda_runtime.h>

#include <cstdint>

#include "ghostz_b200.h"
#include "gzb_common.h"

namespace gzb {

namespace {

constexpr int kTranslateBlock = 256;
constexpr uint8_t kNoBase = 4;
constexpr uint8_t kUnknownCode = 24;  // X in ARNDCQEGHILKMFPSTWYVBJZ*X

// The standard genetic code, codons in ACGT order (first base slowest).
__constant__ char c_codon_letter[65] =
    "KNKNTTTTRSRSIIMIQHQHPPPPRRRRLLLLEDEDAAAAGGGGVVVV*Y*YSSSS*CWCLFLF";
__constant__ char c_protein_letters[26] = "ARNDCQEGHILKMFPSTWYVBJZ*X";

__device__ __forceinline__ uint8_t forward_base(int c) {
  return c == 'A' ? 0 : c == 'C' ? 1 : c == 'G' ? 2 : c == 'T' ? 3 : kNoBase;
}

// the base index of the complement of c
__device__ __forceinline__ uint8_t complement_base(int c) {
  return (c == 'A' || c == 'a')   ? 3
         : (c == 'C' || c == 'c') ? 2
         : (c == 'G' || c == 'g') ? 1
         : (c == 'T' || c == 't') ? 0
                                  : kNoBase;
}

__global__ void __launch_bounds__(kTranslateBlock)
    translate_kernel(const uint8_t *__restrict__ dna, const uint64_t *__restrict__ offsets,
                     const uint32_t *__restrict__ lengths, uint32_t n,
                     const uint64_t *__restrict__ out_offsets, uint8_t delimiter,
                     uint8_t *__restrict__ out) {
  __shared__ uint8_t fwd[256], rev[256], codon[64];
  for (int t = threadIdx.x; t < 256; t += blockDim.x) {
    fwd[t] = forward_base(t);
    rev[t] = complement_base(t);
  }
  if (threadIdx.x < 64) {
    const char l = c_codon_letter[threadIdx.x];
    uint8_t code = kUnknownCode;
    for (int i = 0; i < 25; ++i)
      if (c_protein_letters[i] == l) code = (uint8_t)i;
    codon[threadIdx.x] = code;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += warps) {
    const uint8_t *s = dna + offsets[r];
    const uint32_t len = lengths[r];
    uint8_t *q = out + out_offsets[r];
    if (len < 3) {
      if (lane < 2) q[lane] = delimiter;
      continue;
    }
    const uint32_t slot = len / 3 + 1;
    const uint32_t n0 = len / 3, n1 = (len - 1) / 3, n2 = (len - 2) / 3;  // codons per offset
    if (lane == 0) q[0] = delimiter;
    // lane j: codon j of all six frames (slot position j of each frame)
    for (uint32_t j = lane; j < slot; j += 32) {
      const uint32_t p = 3 * j;
      uint8_t v0 = delimiter, v1 = delimiter, v2 = delimiter;
      uint8_t r0 = delimiter, r1 = delimiter, r2 = delimiter;
      if (j < n0) {
        const uint8_t a = fwd[s[p]], b = fwd[s[p + 1]], c = fwd[s[p + 2]];
        v0 = (a | b | c) & kNoBase ? kUnknownCode : codon[a * 16 + b * 4 + c];
        // the complementary strand's codon j, offset 0: read positions len-1-p ..
        const uint8_t x = rev[s[len - 1 - p]], y = rev[s[len - 2 - p]], z = rev[s[len - 3 - p]];
        r0 = (x | y | z) & kNoBase ? kUnknownCode : codon[x * 16 + y * 4 + z];
      }
      if (j < n1) {
        const uint8_t a = fwd[s[p + 1]], b = fwd[s[p + 2]], c = fwd[s[p + 3]];
        v1 = (a | b | c) & kNoBase ? kUnknownCode : codon[a * 16 + b * 4 + c];
        const uint8_t x = rev[s[len - 2 - p]], y = rev[s[len - 3 - p]], z = rev[s[len - 4 - p]];
        r1 = (x | y | z) & kNoBase ? kUnknownCode : codon[x * 16 + y * 4 + z];
      }
      if (j < n2) {
        const uint8_t a = fwd[s[p + 2]], b = fwd[s[p + 3]], c = fwd[s[p + 4]];
        v2 = (a | b | c) & kNoBase ? kUnknownCode : codon[a * 16 + b * 4 + c];
        const uint8_t x = rev[s[len - 3 - p]], y = rev[s[len - 4 - p]], z = rev[s[len - 5 - p]];
        r2 = (x | y | z) & kNoBase ? kUnknownCode : codon[x * 16 + y * 4 + z];
      }
      uint8_t *f = q + 1 + j;
      f[0] = v0;
      f[slot] = v1;
      f[2 * slot] = v2;
      f[3 * slot] = r0;
      f[4 * slot] = r1;
      f[5 * slot] = r2;
    }
  }
}

}  // namespace

}  // namespace gzb

extern "C" uint64_t gzb_translated_query_length(uint32_t length) {
  return length < 3 ? 2 : 7 + 6 * (uint64_t)(length / 3);
}

extern "C" int gzb_translate_dna_queries(const uint8_t *d_dna, const uint64_t *d_offsets,
                                         const uint32_t *d_lengths, uint32_t number_reads,
                                         const uint64_t *d_out_offsets, uint8_t delimiter,
                                         uint8_t *d_out, void *stream) {
  using namespace gzb;
  if (number_reads == 0) return GZB_OK;
  GZB_CHECK(d_dna && d_offsets && d_lengths && d_out_offsets && d_out, GZB_ERR_INVALID,
            "gzb_translate_dna_queries: null buffer");
  const uint32_t per_block = kTranslateBlock / 32;
  const uint64_t want = (number_reads + per_block - 1) / per_block;
  const uint32_t blocks = (uint32_t)(want < 148u * 16u ? want : 148u * 16u);
  translate_kernel<<<blocks, kTranslateBlock, 0, (cudaStream_t)stream>>>(
      d_dna, d_offsets, d_lengths, number_reads, d_out_offsets, delimiter, d_out);
  GZB_CUDA(cudaGetLastError());
  return GZB_OK;
}
