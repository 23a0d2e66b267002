// CPU check of the host-side record planning (vampire_b200/csrc/record_plan.h):
// builds the SELL-32 layout of a tensor-exchange system the way the uploader
// does, then the compact records and the window plans for tiles of 2, 4 and 8
// slices, and checks every invariant the device passes rely on:
//   * compact word -> neighbour index and dictionary entry {J, d} of the bond;
//   * window segments: 16-byte aligned source (multiple of 4 atoms), length a
//     positive multiple of 4, source range inside the padded state arrays,
//     slots laid end to end inside the tile's slot count, count <= limits;
//   * window word -> slot whose segment maps back to the bond's neighbour,
//     and the bond's dictionary index unchanged.
// Input (binary, little endian): int32 n, M, then int64 nbonds, int32
// nl_start[n], nl_end[n], nl[nbonds], type[n], float64 jlist[9 nbonds].
// Prints "compact <entries>" and one "window sl=<sl> tiles=<t> wmax=<w>
// segs=<s>" line per tile shape ("window sl=<sl> none" when the plan does not
// fit), and exits non-zero at the first violated invariant.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "record_plan.h"

using namespace vgpu;

static void fail(const char* what, long long a, long long b) {
   std::fprintf(stderr, "FAIL %s (%lld, %lld)\n", what, a, b);
   std::exit(1);
}

int main(int argc, char** argv) {
   if (argc < 2) return 2;
   FILE* f = std::fopen(argv[1], "rb");
   if (!f) return 2;
   int32_t n, M;
   int64_t nb;
   if (std::fread(&n, 4, 1, f) != 1 || std::fread(&M, 4, 1, f) != 1 || std::fread(&nb, 8, 1, f) != 1) return 2;
   std::vector<int32_t> st(n), en(n), nl(nb), type(n);
   std::vector<double> J(9 * nb);
   if (std::fread(st.data(), 4, n, f) != (size_t)n || std::fread(en.data(), 4, n, f) != (size_t)n ||
       std::fread(nl.data(), 4, nb, f) != (size_t)nb || std::fread(type.data(), 4, n, f) != (size_t)n ||
       std::fread(J.data(), 8, 9 * nb, f) != (size_t)(9 * nb))
      return 2;
   std::fclose(f);

   // SELL-32 layout and the material-pair table, as the uploader builds them
   const int nslices = (n + 31) / 32;
   const int n_alloc = nslices * 32 + 1, pad = n_alloc - 1, n_alloc4 = (n_alloc + 3) & ~3;
   int shift = 1;
   while ((1 << shift) <= pad) ++shift;
   const int use_shift = M > 1 ? shift : 0;
   std::vector<int> off(nslices + 1, 0);
   for (int s = 0; s < nslices; ++s) {
      int w = 0;
      for (int l = 0; l < 32; ++l)
         if (s * 32 + l < n) w = std::max(w, en[s * 32 + l] - st[s * 32 + l] + 1);
      off[s + 1] = off[s] + 32 * w;
   }
   const size_t ne = (size_t)off[nslices];
   std::vector<int> col(ne, pad);
   std::vector<std::vector<float>> jb(3, std::vector<float>(ne, 0.0f));
   std::vector<float> tabR((size_t)3 * M * M, 0.0f), tabS((size_t)M * M, 0.0f);
   bool scalar = true;
   for (int i = 0; i < n; ++i) {
      int k = 0;
      for (int64_t b = st[i]; b <= en[i]; ++b, ++k) {
         const size_t e = (size_t)off[i >> 5] + 32 * (size_t)k + (i & 31);
         const int j = nl[b];
         col[e] = j | (use_shift ? (type[j] << use_shift) : 0);
         const double* T = &J[9 * b];
         jb[0][e] = (float)T[7]; jb[1][e] = (float)T[2]; jb[2][e] = (float)T[3];
         const size_t pr = (size_t)type[i] * M + type[j];
         tabR[3 * pr] = (float)T[0]; tabR[3 * pr + 1] = (float)T[4]; tabR[3 * pr + 2] = (float)T[8];
         tabS[pr] = (float)T[0];
         if (T[0] != T[4] || T[0] != T[8]) scalar = false;
      }
   }

   std::vector<uint32_t> crec;
   std::vector<float> dict;
   int ndict = 0;
   if (!build_compact_records(off, col, n, type.data(), M, shift, use_shift, jb, scalar, tabS, tabR, crec, dict,
                              ndict)) {
      std::printf("compact none\n");
      return 0;
   }
   std::printf("compact %d\n", ndict);
   const uint32_t jmask = (1u << shift) - 1u;
   const uint32_t cmask = use_shift ? (1u << use_shift) - 1u : 0xffffffffu;
   for (int i = 0; i < n; ++i) {
      int k = 0;
      for (int64_t b = st[i]; b <= en[i]; ++b, ++k) {
         const size_t e = (size_t)off[i >> 5] + 32 * (size_t)k + (i & 31);
         const uint32_t w = crec[e];
         if ((w & jmask) != ((uint32_t)col[e] & cmask)) fail("compact neighbour", (long long)e, w);
         const uint32_t q = w >> shift;
         if ((int)q >= ndict) fail("dictionary index", (long long)e, q);
         const float* A = &dict[4 * q];
         const size_t pr = (size_t)type[i] * M + type[nl[b]];
         if (A[1] != jb[0][e] || A[2] != jb[1][e] || A[3] != jb[2][e]) fail("dictionary d", (long long)e, q);
         if (A[0] != (scalar ? tabS[pr] : tabR[3 * pr])) fail("dictionary J", (long long)e, q);
         if (!scalar) {
            const float* B = &dict[4 * ((size_t)ndict + q)];
            if (B[0] != tabR[3 * pr + 1] || B[1] != tabR[3 * pr + 2]) fail("dictionary diagonal", (long long)e, q);
         }
      }
   }

   for (int sl : {2, 4, 8}) {
      std::vector<uint32_t> lrec;
      std::vector<int4> segs;
      std::vector<int> tseg, tw;
      int wmax = 0;
      if (!build_window_plan(off, crec, shift, sl, nslices, lrec, segs, tseg, tw, wmax)) {
         std::printf("window sl=%d none\n", sl);
         continue;
      }
      const int ntiles = (nslices + sl - 1) / sl;
      if ((int)tseg.size() != ntiles + 1 || tseg[ntiles] != (int)segs.size()) fail("tile segment index", ntiles, 0);
      for (int t = 0; t < ntiles; ++t) {
         int slots = 0;
         if (tseg[t + 1] - tseg[t] > kWindowMaxSegs) fail("segments per tile", t, tseg[t + 1] - tseg[t]);
         for (int g = tseg[t]; g < tseg[t + 1]; ++g) {
            const int4 s = segs[g];
            if (s.x < 0 || s.x % 4 || s.y <= 0 || s.y % 4 || s.x + s.y > n_alloc4) fail("segment source", g, s.x);
            if (s.z != slots) fail("segment slot", g, s.z);
            if (g > tseg[t] && s.x < segs[g - 1].x + segs[g - 1].y) fail("segment order", g, s.x);
            slots += s.y;
         }
         if (slots != tw[t] || slots > kWindowMaxSlots || slots > wmax) fail("tile slots", t, slots);
         const int s0 = t * sl, s1 = std::min(s0 + sl, nslices);
         for (int e = off[s0]; e < off[s1]; ++e) {
            const uint32_t w = lrec[e], slot = w & 0xffffu;
            if ((w >> 16) != (crec[e] >> shift)) fail("window dictionary index", e, w);
            if ((int)slot >= tw[t]) fail("window slot range", e, slot);
            int g = tseg[t];
            while (g + 1 < tseg[t + 1] && segs[g + 1].z <= (int)slot) ++g;
            const uint32_t j = (uint32_t)(segs[g].x + ((int)slot - segs[g].z));
            if (j != (crec[e] & jmask)) fail("window slot maps to neighbour", e, j);
         }
      }
      std::printf("window sl=%d tiles=%d wmax=%d segs=%zu\n", sl, ntiles, wmax, segs.size());
   }
   return 0;
}
