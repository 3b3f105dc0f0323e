// Host-only layout check of the INT8 FP64 matvec kernels (matvec_oz.cuh).
//
// Replays, with the kernels' own constants and offset helpers, every global
// store, bulk copy, shared-memory descriptor range and tensor-memory column
// that oz_digits_kernel, oz_pack_b_kernel and oz_mma_kernel touch for a set of
// problem sizes, and checks each against the buffer sizes the solver
// allocates.  For small sizes it also checks that every byte of the digit
// planes and of the B image is written exactly once (the MMA reads all of
// them).  No CUDA call is made: this runs on a machine without a GPU.
//
// Usage: oz_layout_check   (exit 0: all checks passed)
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "matvec_oz.cuh"

using namespace mbc::oz;

static long fails = 0;
#define CHECK(c, ...)                    \
  do {                                   \
    if (!(c)) {                          \
      if (fails < 20) {                  \
        std::fprintf(stderr, __VA_ARGS__); \
        std::fputc('\n', stderr);        \
      }                                  \
      ++fails;                           \
    }                                    \
  } while (0)

// oz_digits_kernel<DIR> for M outputs and reduction length K, over the row
// tiles [rt0, rt0 + cnt) into a plane buffer of abytes (the whole matrix:
// rt0 = 0, cnt = all tiles; a slab: the slab's tiles at the buffer's start)
static void check_digits(int M, int K, bool full, int rt0 = 0, int cnt = -1, size_t abytes = 0)
{
  const int nks = nks_for(K), nch = nchunks_for(K), nrt = row_tiles(M);
  if (cnt < 0) cnt = nrt;
  if (abytes == 0) abytes = adig_bytes(M, K);
  const size_t ecount = aexp_count(M, K);
  CHECK(cnt <= 65535 && rt0 + cnt <= nrt, "digits: grid.y %d at %d of %d", cnt, rt0, nrt);
  const size_t used = (size_t)cnt * nks * kDigits * kPlaneBytes;  // bytes the launch must fill
  CHECK(used <= abytes, "digits: %zu plane bytes > buffer %zu", used, abytes);
  std::vector<unsigned char> cover(full ? used : 0, 0);
  std::vector<unsigned char> ecover(full && rt0 == 0 && cnt == nrt ? ecount : 0, 0);
  for (int c = 0; c < nch; ++c) {
    for (int rl = 0; rl < cnt; ++rl) {
      const int rt = rt0 + rl;
      if (!full && !(rl == 0 || rl == cnt - 1) && !(c == 0 || c == nch - 1)) continue;
      const int ks0 = c * kChunkSteps, ks1 = std::min(ks0 + kChunkSteps, nks);
      const int kbase = ks0 * kKS, kcount = std::min(kChunk, K - kbase);
      CHECK(kcount > 0 && kbase + kcount <= K, "digits: chunk %d range", c);
      for (int warp = 0; warp < 8; ++warp)
        for (int lane = 0; lane < 32; ++lane) {
          const int sub = lane >> 3, c16 = lane & 7;
          for (int u = 0; u < 4; ++u) {
            const int row = 32 * u + 4 * warp + sub;
            CHECK(row >= 0 && row < kM, "digits: row %d", row);
            const size_t ei = aexp_index(rt, c, row, nch);
            CHECK(ei < ecount, "digits: aexp index %zu >= %zu", ei, ecount);
            if (c16 == 0 && !ecover.empty() && ei < ecount) ++ecover[ei];
            for (int ks = ks0; ks < ks1; ++ks) {
              const int kk0 = (ks - ks0) * kKS + c16 * 16;
              CHECK(kk0 >= 0 && kk0 + 15 < kChunk, "digits: staged index %d", kk0 + 15);
              for (int p = 0; p < kDigits; ++p) {
                const size_t off = adig_offset(rl, ks, 0, nks) + (size_t)p * kPlaneBytes + sw128_i8(row, c16);
                CHECK(off % 16 == 0 && off + 16 <= abytes, "digits: store at %zu (+16) > %zu", off, abytes);
                if (full && off + 16 <= used)
                  for (int b = 0; b < 16; ++b) ++cover[off + b];
              }
            }
          }
        }
    }
  }
  if (full) {
    for (size_t i = 0; i < used; ++i) CHECK(cover[i] == 1, "digits: byte %zu written %d times", i, cover[i]);
    for (size_t i = 0; i < ecover.size(); ++i)
      CHECK(ecover[i] == 1, "digits: exponent %zu written %d times", i, ecover[i]);
  }
}

// oz_pack_b_kernel for reduction length K and R columns
static void check_pack(int K, int R, bool full)
{
  const int np = np_for(R), groups = groups_for(R), nks = nks_for(K), nch = nchunks_for(K);
  const size_t bbytes = bimg_bytes(K, R), ecount = bexp_count(K, R);
  CHECK(np % 16 == 0 && np >= 16 && np <= kNpMax && groups * np >= R, "pack: np %d groups %d R %d", np, groups, R);
  CHECK(groups <= 65535, "pack: grid.y %d", groups);
  std::vector<unsigned char> cover(full ? bbytes : 0, 0);
  std::vector<unsigned char> ecover(full ? ecount : 0, 0);
  for (int c = 0; c < nch; ++c)
    for (int grp = 0; grp < groups; ++grp) {
      const int ks0 = c * kChunkSteps, ks1 = std::min(ks0 + kChunkSteps, nks);
      const int kbase = ks0 * kKS, kcount = std::min(kChunk, K - kbase);
      for (int col = 0; col < np; ++col) {
        const int gc = grp * np + col;
        if (gc < R) CHECK((size_t)(kbase + kcount - 1) * R + gc < (size_t)K * R, "pack: read past vin");
        const size_t ei = bexp_index(grp, c, col, nch, np);
        CHECK(ei < ecount, "pack: bexp index %zu >= %zu", ei, ecount);
        if (full && ei < ecount) ++ecover[ei];
      }
      const int units = (ks1 - ks0) * np * 8;
      for (int t = 0; t < units; ++t) {
        const int col = t % np, rest = t / np, c16 = rest & 7, ks = ks0 + (rest >> 3);
        CHECK(ks < ks1, "pack: k-step %d", ks);
        for (int p = 0; p < kDigits; ++p) {
          const size_t off = bimg_offset(grp, ks, nks, np) + sw128_i8(p * np + col, c16);
          CHECK(sw128_i8(p * np + col, c16) + 16 <= (uint32_t)bstage_bytes(np), "pack: outside the stage");
          CHECK(off % 16 == 0 && off + 16 <= bbytes, "pack: store at %zu (+16) > %zu", off, bbytes);
          if (full && off + 16 <= bbytes)
            for (int b = 0; b < 16; ++b) ++cover[off + b];
        }
      }
    }
  if (full) {
    for (size_t i = 0; i < bbytes; ++i) CHECK(cover[i] == 1, "pack: byte %zu written %d times", i, cover[i]);
    for (size_t i = 0; i < ecount; ++i) CHECK(ecover[i] == 1, "pack: exponent %zu written %d times", i, ecover[i]);
  }
}

// oz_mma_kernel for M outputs, K reduction, R columns; part_rows: rows of the
// curvature-partials buffer the columns direction writes (0: none); a slab
// launch covers row tiles [rt0, rt0 + cnt) with the slab's planes in abytes
static void check_mma(int M, int K, int R, int part_rows, int rt0 = 0, int cnt = -1, size_t abytes = 0)
{
  const int np = np_for(R), groups = groups_for(R), nks = nks_for(K), nch = nchunks_for(K);
  const int nrt_all = row_tiles(M), BST = bstage_bytes(np), TC = tmem_cols_for(np);
  const int nrt = cnt < 0 ? nrt_all : cnt;
  if (abytes == 0) abytes = adig_bytes(M, K);
  const size_t bbytes = bimg_bytes(K, R);
  CHECK(rt0 + nrt <= nrt_all, "mma: slab %d + %d > %d", rt0, nrt, nrt_all);
  CHECK((long long)nrt * groups < (1ll << 31), "mma: grid %d x %d", nrt, groups);
  CHECK(smem_bytes(np) <= kSmemLimit, "mma: shared memory %d", smem_bytes(np));
  CHECK(kPlaneBytes % 1024 == 0 && BST % 1024 == 0, "mma: stage alignment");
  CHECK((2 * kASlots + 2 * kBSlots + 3) * 8 + 4 + 4 + 8 <= 256, "mma: barrier tail");
  CHECK(tail_bytes(np) >= 256 + 4 * np * 8, "mma: partials tail");
  CHECK(TC >= kLevels * np && TC <= 512 && (TC & (TC - 1)) == 0 && TC >= 32, "mma: tensor memory %d", TC);
  CHECK(part_rows == 0 || nrt_all <= part_rows, "mma: partial rows %d > %d", nrt_all, part_rows);
  for (int rt = 0; rt < nrt; ++rt)
    for (int grp = 0; grp < groups; ++grp)
      for (int ks = 0; ks < nks; ++ks) {
        if (rt != 0 && rt != nrt - 1 && ks != 0 && ks != nks - 1) continue;
        const size_t boff = bimg_offset(grp, ks, nks, np);
        CHECK(boff % 16 == 0 && boff + BST <= bbytes, "mma: B copy %zu + %d > %zu", boff, BST, bbytes);
        for (int p = 0; p < kDigits; ++p) {
          const size_t aoff = adig_offset(rt, ks, p, nks);
          CHECK(aoff % 16 == 0 && aoff + kPlaneBytes <= abytes, "mma: A copy %zu > %zu", aoff, abytes);
        }
      }
  // MMA shapes, descriptor ranges and accumulator columns
  for (int p = 0; p < kDigits; ++p) {
    const int nt = np * (kDigits - p);
    for (int kk = 0; kk < kKS / 32; ++kk)
      for (int n0 = 0; n0 < nt; n0 += 256) {
        const int nn = nt - n0 < 256 ? nt - n0 : 256;
        CHECK(nn % 16 == 0 && nn >= 16 && nn <= 256, "mma: N %d", nn);
        CHECK(n0 % 8 == 0 && (n0 + nn) <= kDigits * np, "mma: B rows %d..%d", n0, n0 + nn);
        CHECK((n0 + nn + 7) / 8 * 1024 <= BST, "mma: B descriptor past the stage");
        CHECK(kk * 32 + 32 <= 128, "mma: K offset");
        CHECK(p * np + n0 + nn <= TC, "mma: D columns %d", p * np + n0 + nn);
        // the levels this MMA feeds: B plane q at D column (p + q) np
        CHECK(p * np + n0 >= p * np, "mma: D start");
      }
  }
  const int NPH = np / 2;
  CHECK(NPH % 8 == 0, "acc: columns per warp %d", NPH);
  for (int aw = 0; aw < kAccWarps; ++aw) {
    const int c0 = (aw >> 2) * NPH;
    for (int g = 0; g < NPH / 8; ++g)
      for (int l = 0; l < kLevels; ++l)
        CHECK(l * np + c0 + g * 8 + 8 <= TC, "acc: tensor-memory column %d", l * np + c0 + g * 8 + 8);
    for (int c = 0; c < nch; ++c) {
      CHECK(bexp_index(groups - 1, c, c0 + NPH - 1, nch, np) < bexp_count(K, R), "acc: bexp index");
      CHECK(aexp_index(rt0 + nrt - 1, c, kM - 1, nch) < aexp_count(M, K), "acc: aexp index");
    }
    for (int k = 0; k < NPH; ++k) CHECK((4 - 1) * np + c0 + k < 4 * np, "acc: s_red index");
  }
}

int main()
{
  const int small[][2] = {{1, 1}, {1, 300}, {300, 1}, {127, 129}, {128, 128}, {129, 2047}, {2049, 130}, {3000, 2500}};
  const int Rs[] = {1, 6, 12, 15, 16, 17, 33, 64, 95, 96, 97, 100, 150, 191, 192, 193, 256, 300};
  for (auto &s : small) {
    const int nf = s[0], n = s[1];
    check_digits(nf, n, true);
    check_digits(n, nf, true);
    for (int R : Rs) {
      check_pack(n, R, true);
      check_pack(nf, R, true);
      // the solver sizes the B image for max(n, nf); both directions must fit
      const int K = std::max(n, nf);
      CHECK(bimg_bytes(n, R) <= bimg_bytes(K, R) && bimg_bytes(nf, R) <= bimg_bytes(K, R), "B image sizing");
      CHECK(bexp_count(n, R) <= bexp_count(K, R) && bexp_count(nf, R) <= bexp_count(K, R), "B exponent sizing");
      check_mma(nf, n, R, 0);
      check_mma(n, nf, R, (n + 63) / 64);
    }
  }
  // slab mode: the planes of `per` row tiles at a time in one buffer sized
  // for the larger direction, exponents for every row
  for (auto &s : small) {
    const int nf = s[0], n = s[1];
    for (int per : {1, 2, 3}) {
      const size_t t0 = (size_t)nks_for(n) * kDigits * kPlaneBytes, t1 = (size_t)nks_for(nf) * kDigits * kPlaneBytes;
      const int p0 = std::min(per, row_tiles(nf)), p1 = std::min(per, row_tiles(n));
      const size_t buf = std::max(p0 * t0, p1 * t1);
      for (int r0 = 0; r0 < row_tiles(nf); r0 += p0) {
        const int cnt = std::min(p0, row_tiles(nf) - r0);
        check_digits(nf, n, true, r0, cnt, buf);
        for (int R : {1, 96, 192}) check_mma(nf, n, R, 0, r0, cnt, buf);
      }
      for (int r0 = 0; r0 < row_tiles(n); r0 += p1) {
        const int cnt = std::min(p1, row_tiles(n) - r0);
        check_digits(n, nf, true, r0, cnt, buf);
        for (int R : {1, 96, 192}) check_mma(n, nf, R, (n + 63) / 64, r0, cnt, buf);
      }
    }
  }
  // the large configuration in slabs of a 40 GiB buffer: extremes only
  {
    const int n = 200000;
    const size_t t = (size_t)nks_for(n) * kDigits * kPlaneBytes;
    const int per = (int)std::min<size_t>(row_tiles(n), ((size_t)40 << 30) / t);
    for (int r0 : {0, (row_tiles(n) - 1) / per * per}) {
      const int cnt = std::min(per, row_tiles(n) - r0);
      check_digits(n, n, false, r0, cnt, (size_t)per * t);
      check_mma(n, n, 120, (n + 63) / 64, r0, cnt, (size_t)per * t);
    }
  }
  // full-size shapes: extremes only
  const int big[][2] = {{64000, 64000}, {64000, 32000}, {100003, 77777}};
  for (auto &s : big) {
    check_digits(s[0], s[1], false);
    check_digits(s[1], s[0], false);
    for (int R : {1, 96, 192, 256}) {
      check_pack(s[1], R, false);
      check_mma(s[0], s[1], R, 0);
      check_mma(s[1], s[0], R, (s[1] + 63) / 64);
    }
  }
  if (fails) {
    std::fprintf(stderr, "%ld layout checks failed\n", fails);
    return 1;
  }
  std::printf("all layout checks passed\n");
  return 0;
}
