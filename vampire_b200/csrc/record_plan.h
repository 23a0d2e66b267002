// Host-side planning of the FP32 DMI bond-record layouts (pure C++, no device
// code, so that the plans can be checked on a machine without a GPU):
// compact records with their coupling dictionary, and the window plan of the
// window-staged passes.
#pragma once
#include <stdint.h>
#include <vector_types.h>

#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

namespace vgpu {

constexpr int kDictMax = 512;           // coupling dictionary entries (compact records)
constexpr int kWindowMaxSlots = 4096;   // window slots a tile may take (48 KB of spins)
constexpr int kWindowMaxSegs = 256;     // contiguous segments a tile's window may have
constexpr uint32_t kWindowGap = 8;      // gaps bridged inside one segment (atoms)

inline int4 make_seg(int a, int b, int c) {
   int4 v;
   v.x = a; v.y = b; v.z = c; v.w = 0;
   return v;
}

// Shared-memory bank placement of the coupling dictionary.  A 16-byte load
// by a warp is served a quarter-warp (8 lanes) at a time, and two lanes of a
// quarter that read different entries whose ids are equal modulo 8 fall in
// the same four banks and are served in turn.  The ids are therefore
// reassigned so that entries that quarter-warps read together at the same
// bond slot get different residues modulo 8: the co-reads of every pair of
// entries are counted over the SELL layout, then each entry (heaviest first)
// takes the residue with the least co-read weight to the entries already
// placed there, at most ceil(n / 8) per residue; id = residue + 8 x (its rank
// within the residue).  Ids that no entry takes are left as zero entries.
// Only the placement changes: every bond keeps its coupling values.
inline void bank_order_dictionary(const std::vector<int>& off, int shift, bool scalar, size_t qmax,
                                  std::vector<uint32_t>& crec, std::vector<float>& dict, int& ndict) {
   const int nd = ndict;
   const int cap = (nd + 7) / 8;
   if (8 * (size_t)cap > qmax) return;  // no room for the spread ids: keep first-seen ids
   const int nslices = (int)off.size() - 1;
   const uint32_t low = (1u << shift) - 1u;
   std::vector<double> wgt((size_t)nd * nd, 0.0);
   int q8[8];
   for (int sl = 0; sl < nslices; ++sl) {
      const int w = (off[sl + 1] - off[sl]) >> 5;
      for (int k = 0; k < w; ++k)
         for (int g = 0; g < 4; ++g) {
            int m = 0;
            for (int l = 8 * g; l < 8 * g + 8; ++l) {
               const int q = (int)(crec[(size_t)off[sl] + 32 * (size_t)k + l] >> shift);
               bool seen = false;
               for (int u = 0; u < m; ++u) seen |= q8[u] == q;
               if (!seen) q8[m++] = q;
            }
            for (int u = 0; u < m; ++u)
               for (int v = u + 1; v < m; ++v) {
                  wgt[(size_t)q8[u] * nd + q8[v]] += 1.0;
                  wgt[(size_t)q8[v] * nd + q8[u]] += 1.0;
               }
         }
   }
   std::vector<int> order(nd), res(nd, -1), count(8, 0), rank(nd, 0);
   std::vector<double> tot(nd, 0.0);
   for (int a = 0; a < nd; ++a) {
      order[a] = a;
      for (int b = 0; b < nd; ++b) tot[a] += wgt[(size_t)a * nd + b];
   }
   std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return tot[x] > tot[y]; });
   for (int a : order) {
      int best = -1;
      double bw = 0.0;
      for (int r = 0; r < 8; ++r) {
         if (count[r] >= cap) continue;
         double c = 0.0;
         for (int b = 0; b < nd; ++b)
            if (res[b] == r) c += wgt[(size_t)a * nd + b];
         if (best < 0 || c < bw) { best = r; bw = c; }
      }
      res[a] = best;
      rank[a] = count[best]++;
   }
   const int nnew = 8 * cap;
   std::vector<uint32_t> id(nd);
   for (int a = 0; a < nd; ++a) id[a] = (uint32_t)(res[a] + 8 * rank[a]);
   for (auto& wd : crec) wd = (wd & low) | (id[wd >> shift] << shift);
   const int blocks = scalar ? 1 : 2;  // {J, d} entries, then {Jyy, Jzz} entries
   std::vector<float> out((size_t)4 * nnew * blocks, 0.0f);
   for (int bl = 0; bl < blocks; ++bl)
      for (int a = 0; a < nd; ++a)
         for (int c = 0; c < 4; ++c) out[4 * ((size_t)bl * nnew + id[a]) + c] = dict[4 * ((size_t)bl * nd + a) + c];
   dict.swap(out);
   ndict = nnew;
}

// Compact FP32 DMI records: every SELL entry e becomes the word
// j | q << shift, q indexing a dictionary of the distinct couplings
// {J (or Jxx), d_x, d_y, d_z} (+ {Jyy, Jzz, 0, 0} for a non-scalar diagonal),
// keyed by (own material, neighbour material, d): the values the 16-byte
// records and the material table give the same bond, so the passes compute
// the same field.  Padding entries key as (own material, 0, d = 0), as their
// 16-byte records read.  Returns false (no compact records) when the distinct
// couplings exceed kDictMax or the index bits left above the neighbour index.
struct DictKey {
   int mi, mj;
   uint32_t d[3];
};
inline bool build_compact_records(const std::vector<int>& off, const std::vector<int>& col, int n, const int* type,
                                  int M, int shift, int use_shift, const std::vector<std::vector<float>>& jb,
                                  bool scalar, const std::vector<float>& tabS, const std::vector<float>& tabR,
                                  std::vector<uint32_t>& crec, std::vector<float>& dict, int& ndict) {
   const int nslices = (int)off.size() - 1;
   const int qbits = 32 - shift;
   const size_t qmax = std::min<size_t>(kDictMax, qbits >= 31 ? (size_t)1 << 30 : (size_t)1 << qbits);
   // open-addressing table of dictionary ids (4 x kDictMax slots)
   const size_t cap = 4 * kDictMax;
   std::vector<DictKey> keys;
   std::vector<int> slot(cap, -1);
   std::vector<float> A, B;
   crec.assign(col.size(), 0u);
   const uint32_t jmask = use_shift ? (1u << use_shift) - 1u : 0xffffffffu;
   // ids in first-seen order walking bond slot k, then lane: the couplings one
   // warp reads at the same k get consecutive ids, so its 16-byte dictionary
   // loads fall in distinct shared-memory banks
   for (int sl = 0; sl < nslices; ++sl) {
      const int w = (off[sl + 1] - off[sl]) >> 5;
      for (int k = 0; k < w; ++k) {
         for (int l = 0; l < 32; ++l) {
            const int i = sl * 32 + l;
            const int mi = i < n ? type[i] : 0;
            const size_t e = (size_t)off[sl] + 32 * (size_t)k + l;
            const uint32_t c = (uint32_t)col[e];
            DictKey key{mi, use_shift ? (int)(c >> use_shift) : 0, {0, 0, 0}};
            for (int q = 0; q < 3; ++q) std::memcpy(&key.d[q], &jb[q][e], 4);
            uint64_t hsh = 1469598103934665603ull;
            const uint32_t words[5] = {(uint32_t)key.mi, (uint32_t)key.mj, key.d[0], key.d[1], key.d[2]};
            for (uint32_t v : words) hsh = (hsh ^ v) * 1099511628211ull;
            size_t at = (size_t)(hsh % cap);
            int id = -1;
            while (slot[at] >= 0) {
               const DictKey& o = keys[slot[at]];
               if (o.mi == key.mi && o.mj == key.mj && o.d[0] == key.d[0] && o.d[1] == key.d[1] && o.d[2] == key.d[2]) {
                  id = slot[at];
                  break;
               }
               at = (at + 1) % cap;
            }
            if (id < 0) {
               if (keys.size() >= qmax) return false;
               id = (int)keys.size();
               keys.push_back(key);
               slot[at] = id;
               const size_t pr = (size_t)key.mi * M + key.mj;
               A.push_back(scalar ? tabS[pr] : tabR[3 * pr]);
               A.push_back(jb[0][e]); A.push_back(jb[1][e]); A.push_back(jb[2][e]);
               B.push_back(tabR[3 * pr + 1]); B.push_back(tabR[3 * pr + 2]); B.push_back(0.0f); B.push_back(0.0f);
            }
            crec[e] = (c & jmask) | ((uint32_t)id << shift);
         }
      }
   }
   ndict = (int)keys.size();
   dict = A;
   if (!scalar) dict.insert(dict.end(), B.begin(), B.end());
   if (ndict > 0) bank_order_dictionary(off, shift, scalar, qmax, crec, dict, ndict);
   return ndict > 0;
}

// Window plan of the window-staged passes: for every tile of sl slices, the
// sorted distinct neighbours of its bonds merged into contiguous segments
// (gaps of up to kWindowGap atoms bridged; ends rounded out to 4 atoms, so
// every segment is a 16-byte aligned whole number of 16-byte groups), laid end
// to end as the tile's window slots; each bond's word becomes
// slot | coupling index << 16.  Tiles are planned in parallel on the host.
// Returns false when a tile needs more than kWindowMaxSlots slots or
// kWindowMaxSegs segments (the passes then stay on compact records).
inline bool build_window_plan(const std::vector<int>& off, const std::vector<uint32_t>& crec, int shift, int sl,
                              int nslices_upd, std::vector<uint32_t>& lrec, std::vector<int4>& segs,
                              std::vector<int>& tseg, std::vector<int>& tw, int& wmax) {
   const uint32_t jmask = (1u << shift) - 1u;
   const int ntiles = (nslices_upd + sl - 1) / sl;
   lrec.assign(crec.size(), 0u);
   tw.assign(ntiles, 0);
   int nth = (int)std::thread::hardware_concurrency();
   nth = std::max(1, std::min({nth, 32, ntiles}));
   std::vector<std::vector<int4>> part(nth);
   std::vector<std::vector<int>> pcount(nth);
   std::vector<char> ok(nth, 1);
   auto work = [&](int w) {
      const int t0 = (int)((int64_t)ntiles * w / nth), t1 = (int)((int64_t)ntiles * (w + 1) / nth);
      std::vector<uint32_t> js;
      std::vector<int4>& out = part[w];
      for (int t = t0; t < t1; ++t) {
         const int s0 = t * sl, s1 = std::min(s0 + sl, nslices_upd);
         const int e0 = off[s0], e1 = off[s1];
         js.clear();
         for (int e = e0; e < e1; ++e) js.push_back(crec[e] & jmask);
         std::sort(js.begin(), js.end());
         js.erase(std::unique(js.begin(), js.end()), js.end());
         const size_t first = out.size();
         int slots = 0;
         for (size_t u = 0; u < js.size();) {
            const uint32_t a0 = js[u] & ~3u;
            uint32_t end = js[u] + 1;
            size_t v = u + 1;
            while (v < js.size() && js[v] <= end + kWindowGap) end = js[v++] + 1;
            const uint32_t e4 = (end + 3u) & ~3u;
            out.push_back(make_seg((int)a0, (int)(e4 - a0), slots));
            slots += (int)(e4 - a0);
            u = v;
         }
         if (slots > kWindowMaxSlots || out.size() - first > (size_t)kWindowMaxSegs) {
            ok[w] = 0;
            return;
         }
         pcount[w].push_back((int)(out.size() - first));
         tw[t] = slots;
         for (int e = e0; e < e1; ++e) {
            const uint32_t j = crec[e] & jmask;
            // last segment starting at or below j
            size_t lo = first, hi = out.size();
            while (hi - lo > 1) {
               const size_t mid = (lo + hi) / 2;
               if ((uint32_t)out[mid].x <= j) lo = mid; else hi = mid;
            }
            const uint32_t slot = (uint32_t)out[lo].z + (j - (uint32_t)out[lo].x);
            lrec[e] = slot | ((crec[e] >> shift) << 16);
         }
      }
   };
   std::vector<std::thread> pool;
   for (int w = 1; w < nth; ++w) pool.emplace_back(work, w);
   work(0);
   for (auto& th : pool) th.join();
   for (int w = 0; w < nth; ++w)
      if (!ok[w]) return false;
   segs.clear();
   tseg.assign(ntiles + 1, 0);
   int t = 0;
   for (int w = 0; w < nth; ++w) {
      segs.insert(segs.end(), part[w].begin(), part[w].end());
      for (int c : pcount[w]) { tseg[t + 1] = tseg[t] + c; ++t; }
   }
   wmax = 0;
   for (int x : tw) wmax = std::max(wmax, x);
   return t == ntiles;
}

}  // namespace vgpu
