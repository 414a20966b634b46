/*
 * trellis.c — the §13 trellis coefficient quantiser of the reference
 * encoder (oxideav-vp8 src/encoder.rs), restated for the oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see vp8a_oracle.h).
 *
 *   TRELLIS_LAMBDA_SCALE, TrellisStrength     src/encoder.rs:2654-2711
 *   IDCT_BASIS_NORM_SQ                        src/encoder.rs:2763-2777
 *   coeff_token_bits, eob_token_bits          src/encoder.rs:2789-2831
 *   level_ctx3                                src/encoder.rs:2834-2841
 *   trellis_quantize_block                    src/encoder.rs:3095-3129
 *   trellis_scan_direct                       src/encoder.rs:3468-3582
 *   rounded_level                             src/encoder.rs:3608-3615
 *   MbRdCtx::trellis_lambda                   src/encoder.rs:3661-3664
 *
 * Every call site on the inter path (transform_whole_block_luma_rd
 * :3815-3880, transform_chroma_plane_rd :4133-4170,
 * transform_split_mv_mb_rd :8259-8300) quantises each block on its own
 * with entry context 0, against the frame's coefficient probabilities (the
 * §13.5 defaults when no update is shipped), at lambda = rd_lambda(factors)
 * * (strength * TRELLIS_LAMBDA_SCALE). The direct scan is the listing the
 * reference's tabled production form is pinned against
 * (trellis_lut_and_early_exit_match_reference): the same f64 expressions in
 * the same order.
 */
#include <math.h>
#include <stdatomic.h>
#include <string.h>

#pragma GCC diagnostic ignored "-Wunused-const-variable"
#include "vp8_tables.h"
#include "vp8a_oracle.h"

double vo_bool_bits(uint8_t prob, int value);
#define BB(p, v) vo_bool_bits((uint8_t)(p), (v))

static double g_norm[16];
static atomic_int g_norm_ready;

/* IDCT_BASIS_NORM_SQ: the energy of the §14.4 inverse DCT of a 256 impulse
 * at raster ZIGZAG[k], over 256^2. */
const double* vo_idct_basis_norm_sq(void) {
  if (!atomic_load(&g_norm_ready)) {
    double t[16];
    for (int k = 0; k < 16; k++) {
      int16_t in[16], out[16];
      memset(in, 0, sizeof in);
      in[VO_ZIGZAG[k]] = 256;
      vo_inverse_dct_4x4(in, out);
      double e = 0.0;
      for (int i = 0; i < 16; i++) e += pow((double)out[i], 2.0);
      t[k] = e / pow(256.0, 2.0);
    }
    memcpy(g_norm, t, sizeof t);
    atomic_store(&g_norm_ready, 1);
  }
  return g_norm;
}

/* The §13.2 token of an absolute level: DCT_0..DCT_4 = 0..4, then the
 * extra-bit categories cat1..cat6 = 5..10. */
static int token_of(uint32_t a) {
  if (a <= 4) return (int)a;
  if (a <= 6) return 5;
  if (a <= 10) return 6;
  if (a <= 18) return 7;
  if (a <= 34) return 8;
  if (a <= 66) return 9;
  return 10;
}

/* Each token's path through the §13.2 coefficient tree from the root:
 * (probability index, bit) steps. The first step is the "not EOB" branch,
 * skipped when the previous token was DCT_0. */
static const uint8_t PATH_LEN[11] = {2, 3, 5, 6, 6, 6, 6, 7, 7, 7, 7};
static const uint8_t PATH[11][7][2] = {
    {{0, 1}, {1, 0}},
    {{0, 1}, {1, 1}, {2, 0}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 0}, {4, 0}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 0}, {4, 1}, {5, 0}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 0}, {4, 1}, {5, 1}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 1}, {6, 0}, {7, 0}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 1}, {6, 0}, {7, 1}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 1}, {6, 1}, {8, 0}, {9, 0}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 1}, {6, 1}, {8, 0}, {9, 1}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 1}, {6, 1}, {8, 1}, {10, 0}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 1}, {6, 1}, {8, 1}, {10, 1}},
};

/* coeff_token_bits (src/encoder.rs:2789-2817). */
double vo_coeff_token_bits(int plane, int i, int ctx3, int prev_was_zero, uint32_t level) {
  const uint8_t* probs = VO_DEFAULT_COEF_PROBS[plane][VO_COEFF_BANDS[i]][ctx3];
  const int token = token_of(level);
  double bits = 0.0;
  for (int s = prev_was_zero ? 1 : 0; s < PATH_LEN[token]; s++) bits += BB(probs[PATH[token][s][0]], PATH[token][s][1]);
  if (token >= 5) {
    const int cat = token - 5;
    const uint32_t extra = level - VO_CAT_BASE[cat];
    const int n = VO_PCAT_LEN[cat];
    for (int j = 0; j < n; j++) bits += BB(VO_PCAT[cat][j], (int)((extra >> (n - 1 - j)) & 1u));
  }
  if (level != 0) bits += BB(128, 0);
  return bits;
}

/* eob_token_bits (src/encoder.rs:2825-2831). */
double vo_eob_token_bits(int plane, int i, int ctx3) {
  return BB(VO_DEFAULT_COEF_PROBS[plane][VO_COEFF_BANDS[i]][ctx3][0], 0);
}

static inline int level_ctx3(uint32_t a) { return a == 0 ? 0 : (a == 1 ? 1 : 2); }

/* enc_round_div (src/encoder.rs:2112-2122). */
static int16_t round_div(int32_t num, int32_t den) {
  int32_t a = num < 0 ? -num : num;
  int32_t q = (a + den / 2) / den;
  return (int16_t)(num < 0 ? -q : q);
}

/* trellis_quantize_block with the direct scan (src/encoder.rs:3095-3129,
 * :3468-3582): `block` (raster order, the forward transform's output) is
 * replaced by the chosen levels. lambda <= 0 is plain rounding from
 * first_coeff (enc_quantize_block_range, :3621-3633). */
void vo_trellis_quantize_block(int16_t* block, int16_t dc, int16_t ac, int first_coeff, int entry_ctx3, int plane,
                               double lambda) {
  if (lambda <= 0.0) {
    block[0] = first_coeff == 0 ? round_div(block[0], dc) : 0;
    for (int k = 1; k < 16; k++) block[k] = round_div(block[k], ac);
    return;
  }
  const double* norms = vo_idct_basis_norm_sq();
  const uint32_t dc_q = (uint32_t)dc, ac_q = (uint32_t)ac;
  /* TrellisScan::new (:3150-3172). */
  uint32_t ax[16] = {0}, m_rounds[16] = {0};
  int negative[16] = {0};
  double zero_dist[16] = {0}, suffix[17] = {0};
  int last = -1;
  for (int k = 15; k >= first_coeff; k--) {
    const int16_t x = block[VO_ZIGZAG[k]];
    const uint32_t q = k == 0 ? dc_q : ac_q;
    ax[k] = (uint32_t)(x < 0 ? -(int32_t)x : x);
    negative[k] = x < 0;
    m_rounds[k] = (ax[k] + q / 2) / q; /* rounded_level */
    if (m_rounds[k] != 0 && last < 0) last = k;
    zero_dist[k] = norms[k] * (double)((uint64_t)ax[k] * ax[k]);
    suffix[k] = suffix[k + 1] + zero_dist[k];
  }
  if (last < 0) {
    memset(block, 0, 16 * sizeof(int16_t));
    return;
  }
  double surv_cost[3] = {INFINITY, INFINITY, INFINITY};
  int surv_pwz[3] = {0, 0, 0};
  surv_cost[entry_ctx3] = 0.0;
  uint16_t choice_level[16][3];
  uint8_t choice_prev[16][3];
  memset(choice_level, 0, sizeof choice_level);
  memset(choice_prev, 0, sizeof choice_prev);
  const double entry_eob = vo_eob_token_bits(plane, first_coeff, entry_ctx3);
  double best_term_cost = 0.0 + lambda * entry_eob + suffix[first_coeff];
  int best_term_pos = -1, best_term_ctx = entry_ctx3;
  for (int k = first_coeff; k <= last; k++) {
    const uint32_t m = m_rounds[k];
    const uint32_t q = k == 0 ? dc_q : ac_q;
    const uint32_t cands[3] = {m, m > 0 ? m - 1 : 0, 0};
    const int ncand = (int)(m < 2 ? m : 2) + 1;
    double cand_dist[3] = {0.0, 0.0, 0.0};
    for (int c = 0; c < ncand; c++) {
      if (cands[c] == 0) {
        cand_dist[c] = zero_dist[k];
      } else {
        const int64_t err = (int64_t)ax[k] - (int64_t)cands[c] * (int64_t)q;
        cand_dist[c] = norms[k] * (double)(err * err);
      }
    }
    double next_cost[3] = {INFINITY, INFINITY, INFINITY};
    int next_pwz[3] = {0, 0, 0};
    uint16_t next_level[3] = {0, 0, 0};
    uint8_t next_prev[3] = {0, 0, 0};
    for (int in_ctx = 0; in_ctx < 3; in_ctx++) {
      const double base = surv_cost[in_ctx];
      if (base >= INFINITY) continue;
      const int pwz = surv_pwz[in_ctx];
      for (int c = 0; c < ncand; c++) {
        const uint32_t level = cands[c];
        const double r = vo_coeff_token_bits(plane, k, in_ctx, pwz, level);
        const double cost = base + cand_dist[c] + lambda * r;
        const int out_ctx = level_ctx3(level);
        if (cost < next_cost[out_ctx]) {
          next_cost[out_ctx] = cost;
          next_pwz[out_ctx] = level == 0;
          next_level[out_ctx] = (uint16_t)level;
          next_prev[out_ctx] = (uint8_t)in_ctx;
        }
      }
    }
    memcpy(choice_level[k], next_level, sizeof next_level);
    memcpy(choice_prev[k], next_prev, sizeof next_prev);
    for (int out_ctx = 1; out_ctx < 3; out_ctx++) {
      const double cost = next_cost[out_ctx];
      if (cost >= INFINITY) continue;
      const double term_cost =
          k + 1 < 16 ? cost + lambda * vo_eob_token_bits(plane, k + 1, out_ctx) + suffix[k + 1] : cost;
      if (term_cost < best_term_cost) {
        best_term_cost = term_cost;
        best_term_pos = k;
        best_term_ctx = out_ctx;
      }
    }
    memcpy(surv_cost, next_cost, sizeof next_cost);
    memcpy(surv_pwz, next_pwz, sizeof next_pwz);
  }
  memset(block, 0, 16 * sizeof(int16_t));
  if (best_term_pos >= 0) {
    int k = best_term_pos, ctx = best_term_ctx;
    for (;;) {
      const int16_t level = (int16_t)choice_level[k][ctx];
      block[VO_ZIGZAG[k]] = negative[k] ? (int16_t)-level : level;
      if (k == first_coeff) break;
      ctx = choice_prev[k][ctx];
      k--;
    }
  }
}

/* MbRdCtx::trellis_lambda for a factor set (y1_ac first, as rd_lambda,
 * src/encoder.rs:3742) and a strength already clamped to 0..=8. */
double vo_trellis_lambda(int16_t y1_ac, double strength) {
  const double q = (double)y1_ac;
  const double lambda = q * q / 32.0;
  return lambda * (strength * 0.04);
}
