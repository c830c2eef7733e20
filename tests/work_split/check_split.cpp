// Host-side check of the pair kernel's work-list split (bnb::work_split and
// bnb::work_walk, the functions the list rebuild runs on the device): for
// every candidate count, tile count per item and tail length, the items of a
// block cover its candidates once and in order, level by level, with item
// sizes that never grow from one level to the next, and the per-level counts
// that the rebuild reserves match the items written.  Prints "ok" or the
// first failing case.
#include <cstdio>
#include <vector>

#include "work_split.h"

int main() {
  const int tails[] = {0, 1, 2, 4, 8};
  for (int T = 1; T <= 32; T++)
    for (int tail : tails)
      for (int nc = 0; nc <= 400; nc++) {
        int tiles[bnb::kWorkLevels], items[bnb::kWorkLevels];
        const int L = bnb::work_split(nc, T, tail * T, tiles, items);
        int sumTiles = 0;
        for (int l = 0; l < bnb::kWorkLevels; l++) sumTiles += tiles[l];
        const int K = nc < tail * T ? nc : tail * T;
        if (sumTiles != nc || tiles[0] != nc - K || L < 1 || L > bnb::kWorkLevels) {
          std::printf("split T=%d tail=%d nc=%d: tiles %d head %d L %d\n", T, tail, nc, sumTiles, tiles[0], L);
          return 1;
        }
        const int c0 = 1000;
        int next = c0, lastLevel = 0, lastSize = 1 << 30;
        std::vector<int> count(bnb::kWorkLevels, 0);
        bool bad = false;
        bnb::work_walk(c0, nc, T, tail * T, [&](int l, int k, int first, int n) {
          const int size = bnb::work_item_size(T, l);
          if (first != next || n < 1 || n > size || l < lastLevel || k != count[l] || size > lastSize) bad = true;
          next = first + n;
          if (l != lastLevel) lastSize = bnb::work_item_size(T, lastLevel);
          lastLevel = l;
          count[l]++;
        });
        for (int l = 0; l < bnb::kWorkLevels; l++)
          if (count[l] != items[l]) bad = true;
        if (bad || next != c0 + nc) {
          std::printf("walk T=%d tail=%d nc=%d\n", T, tail, nc);
          return 1;
        }
      }
  std::printf("ok\n");
  return 0;
}
