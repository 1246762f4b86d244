// Seeded synthetic spatial workloads.  The reference's real workload (FPGA
// routing-contest artifacts) is not available, so graphs with the shapes the
// benchmark configurations describe are generated here: a grid of tiles,
// intra-tile edges to uniform nodes of the own tile, inter-tile edges to a
// uniform 4-neighbour tile at a uniform span, uint or log-normal float costs.
//
// PRNG: xoshiro256** (Blackman & Vigna) seeded through splitmix64; uniform
// integers by the multiply-shift reduction of the top 32 bits; standard
// normals by Box-Muller in double precision, rounded once to float.
#include "bfx_host.h"
#include "bfx_internal.hpp"

#include <cmath>
#include <cstring>

namespace bfx {
namespace {

struct Xoshiro256ss {
  std::uint64_t s[4];

  explicit Xoshiro256ss(std::uint64_t seed) {
    std::uint64_t x = seed;
    for (auto& w : s) {
      x += 0x9E3779B97F4A7C15ULL;  // splitmix64 increment
      std::uint64_t z = x;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
      w = z ^ (z >> 31);
    }
  }
  static std::uint64_t rotl(std::uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
  std::uint64_t next() {
    const std::uint64_t result = rotl(s[1] * 5, 7) * 9;
    const std::uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return result;
  }
  std::uint32_t below(std::uint32_t n) {
    return static_cast<std::uint32_t>(((next() >> 32) * static_cast<std::uint64_t>(n)) >> 32);
  }
  double unit() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
  double normal() {
    const double u1 = 1.0 - unit();  // (0, 1]
    const double u2 = unit();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586476925 * u2);
  }
};

void tile_shape(std::uint32_t n, std::uint32_t& sx, std::uint32_t& sy) {
  if (n == 128U) {
    sx = 16U;
    sy = 8U;
    return;
  }
  std::uint32_t s = static_cast<std::uint32_t>(std::lround(std::sqrt(static_cast<double>(n))));
  if (s * s == n) {
    sx = sy = s;
    return;
  }
  sx = n;
  sy = 1U;
}

void check_config(const bfx_synth_config& c) {
  require(c.tiles_x > 0 && c.tiles_y > 0 && c.nodes_per_tile > 0, "empty synthetic grid");
  require(c.intra_degree + c.inter_degree > 0, "synthetic degree must be positive");
  require(c.inter_degree == 0 || (c.span_count > 0 && c.span_count <= 8), "span_count must be 1..8");
  require(c.cost_kind <= 1U, "cost_kind must be 0 or 1");
  require(c.cost_kind != 0U || c.cost_lo <= c.cost_hi, "cost_lo must be <= cost_hi");
  require(c.nodes_per_tile >= 2 || c.intra_degree == 0, "intra edges need two nodes per tile");
  const std::uint64_t V = static_cast<std::uint64_t>(c.tiles_x) * c.tiles_y * c.nodes_per_tile;
  const std::uint64_t E = V * (c.intra_degree + c.inter_degree);
  if (V > 0xFFFFFFFFULL || E > 0xFFFFFFFFULL) throw std::overflow_error("synthetic graph exceeds 32-bit counts");
}

}  // namespace
}  // namespace bfx

extern "C" {

int bfx_synth_sizes(const bfx_synth_config* config, uint64_t out[2]) {
  return bfx::guarded([&] {
    bfx::require(config && out, "null argument");
    bfx::check_config(*config);
    const std::uint64_t V = static_cast<std::uint64_t>(config->tiles_x) * config->tiles_y * config->nodes_per_tile;
    out[0] = V;
    out[1] = V * (config->intra_degree + config->inter_degree);
  });
}

int bfx_synth_fill(const bfx_synth_config* config, int32_t* x, int32_t* y, uint8_t* has_location,
                   uint16_t* resource_class, uint32_t* edge_source, uint32_t* edge_destination,
                   float* edge_weight, uint32_t* provenance_domain, uint32_t* provenance_kind,
                   uint64_t* provenance_record, bfx_spatial_order_config* order, uint64_t stats[2]) {
  return bfx::guarded([&] {
    bfx::require(config && x && y && has_location && resource_class && edge_source && edge_destination &&
                     edge_weight && provenance_domain && provenance_kind && provenance_record && order,
                 "null argument");
    const bfx_synth_config& c = *config;
    bfx::check_config(c);
    std::uint32_t sx = 0, sy = 0;
    bfx::tile_shape(c.nodes_per_tile, sx, sy);
    const std::uint32_t n = c.nodes_per_tile;
    const std::uint32_t TX = c.tiles_x, TY = c.tiles_y;
    bfx::Xoshiro256ss rng(c.seed);
    std::uint64_t e = 0, inter = 0, redrawn = 0;
    auto cost = [&](int span_index) -> float {
      if (c.cost_kind == 0U) {
        return static_cast<float>(c.cost_lo + rng.below(c.cost_hi - c.cost_lo + 1U));
      }
      const double base = span_index < 0 ? c.intra_base : c.span_base[span_index];
      return static_cast<float>(base * std::exp(static_cast<double>(c.sigma) * rng.normal()));
    };
    static const int dxs[4] = {1, -1, 0, 0};
    static const int dys[4] = {0, 0, 1, -1};
    for (std::uint32_t ty = 0; ty < TY; ++ty) {
      for (std::uint32_t tx = 0; tx < TX; ++tx) {
        const std::uint32_t t = ty * TX + tx;
        for (std::uint32_t i = 0; i < n; ++i) {
          const std::uint32_t v = t * n + i;
          x[v] = static_cast<int32_t>(tx * sx + i % sx);
          y[v] = static_cast<int32_t>(ty * sy + i / sx);
          has_location[v] = 1U;
          resource_class[v] = 1U;
          for (std::uint32_t j = 0; j < c.intra_degree; ++j) {
            std::uint32_t r = rng.below(n - 1U);
            if (r >= i) ++r;
            edge_source[e] = v;
            edge_destination[e] = t * n + r;
            edge_weight[e] = cost(-1);
            provenance_domain[e] = 1U;  // provenance_domain::synthetic
            provenance_kind[e] = 1U;    // provenance_kind::synthetic_edge
            provenance_record[e] = e;
            ++e;
          }
          for (std::uint32_t j = 0; j < c.inter_degree; ++j) {
            std::int64_t ntx = 0, nty = 0;
            std::uint32_t span_index = 0;
            bool ok = false;
            for (int attempt = 0; attempt < 16 && !ok; ++attempt) {
              if (attempt > 0) ++redrawn;
              const std::uint32_t d = rng.below(4U);
              span_index = rng.below(c.span_count);
              const std::int64_t span = c.spans[span_index];
              ntx = static_cast<std::int64_t>(tx) + dxs[d] * span;
              nty = static_cast<std::int64_t>(ty) + dys[d] * span;
              ok = ntx >= 0 && nty >= 0 && ntx < TX && nty < TY;
            }
            if (!ok) {  // clamp to the border after 16 draws
              ntx = std::min<std::int64_t>(std::max<std::int64_t>(ntx, 0), TX - 1);
              nty = std::min<std::int64_t>(std::max<std::int64_t>(nty, 0), TY - 1);
            }
            const std::uint32_t nt = static_cast<std::uint32_t>(nty) * TX + static_cast<std::uint32_t>(ntx);
            edge_source[e] = v;
            edge_destination[e] = nt * n + rng.below(n);
            edge_weight[e] = cost(static_cast<int>(span_index));
            provenance_domain[e] = 1U;
            provenance_kind[e] = 1U;
            provenance_record[e] = e;
            ++e;
            ++inter;
          }
        }
      }
    }
    order->origin_x = 0;
    order->origin_y = 0;
    order->tile_width = sx;
    order->tile_height = sy;
    if (stats) {
      stats[0] = inter;
      stats[1] = redrawn;
    }
  });
}

}  // extern "C"
