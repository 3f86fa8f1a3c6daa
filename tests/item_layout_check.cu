// Exhaustive check of the equal-length work-queue layout (UniformB): every
// chunk item appears exactly once, every FIN once and after its row's chunks.
#include "radik_common.cuh"
#include <cstdio>
#include <vector>
using namespace radik;
int main() {
  int bad = 0, cases = 0;
  for (int B : {1, 2, 3, 5, 17, 40, 256})
    for (int nc : {0, 1, 3, 8})
      for (int mult : {1, 2, 3})
        for (int R : {0, 1, 2, 7, 300})
          for (int f : {0, 1})
            for (int D : {1, 2, 5, 28, 400}) {
              if (nc == 0 && f == 0) continue;
              const int nct = nc * mult;
              const int RR = nc == 0 ? 0 : std::min(R, B);
              UniformB u{B, nc, nct, RR, f, D};
              const long long N = u.count();
              std::vector<std::vector<int>> seen(B);
              std::vector<long long> fin_at(B, -1), last_chunk(B, -1);
              for (int r = 0; r < B; ++r) seen[r].assign(u.chunks(r), 0);
              for (long long j = 0; j < N; ++j) {
                int row, sub, fin;
                u.decode(j, &row, &sub, &fin);
                if (row < 0 || row >= B) { ++bad; continue; }
                if (fin) { if (fin_at[row] >= 0) ++bad; fin_at[row] = j; }
                else { if (sub < 0 || sub >= u.chunks(row) || seen[row][sub]) ++bad; else seen[row][sub] = 1; last_chunk[row] = j; }
              }
              for (int r = 0; r < B; ++r) {
                for (int c : seen[r]) if (!c) ++bad;
                if (f && (fin_at[r] < 0 || fin_at[r] < last_chunk[r])) ++bad;
                if (!f && fin_at[r] >= 0) ++bad;
                if (u.chunks(r) > 0) { int row, sub, fin; u.decode(u.first(r), &row, &sub, &fin); if (row != r || sub != 0 || fin) ++bad; }
              }
              ++cases;
            }
  printf("cases %d bad %d\n", cases, bad);
  return bad != 0;
}
