// Split of the pair kernel's work list into levels (no CUDA dependencies, so
// the host-side check in tests/work_split compiles it with a plain C++
// compiler).
#pragma once

#ifdef __CUDACC__
#define BNB_HD __host__ __device__
#else
#define BNB_HD
#endif

namespace bnb {

constexpr int kWorkLevels = 8;  // levels of the work list: items of T, T/2, ..., 1 tiles (T <= 32)

// Split of one i block's nc candidate tiles into work items.  Level 0 takes
// the first nc - K tiles (K = min(nc, tailTiles)) in items of T tiles; the
// last K tiles form the tail, which levels 1, 2, ... take from the front in
// two items each of max(1, T >> level) tiles, the level of 1-tile items
// taking the rest.  tiles[l] and items[l] are per level; returns the number
// of levels used.  The split depends on the block's own count only.
BNB_HD inline int work_split(int nc, int T, int tailTiles, int *tiles, int *items) {
  const int K = nc < tailTiles ? nc : tailTiles;
  tiles[0] = nc - K;
  items[0] = (tiles[0] + T - 1) / T;
  int rest = K, l = 1;
  for (; l < kWorkLevels; l++) {
    const int size = (T >> l) > 1 ? (T >> l) : 1;
    const int take = size == 1 || l == kWorkLevels - 1 ? rest : (rest < 2 * size ? rest : 2 * size);
    tiles[l] = take;
    items[l] = (take + size - 1) / size;
    rest -= take;
    if (size == 1) { l++; break; }
  }
  for (int k = l; k < kWorkLevels; k++) tiles[k] = items[k] = 0;
  return l;
}

// Tile size of the items of a level.
BNB_HD inline int work_item_size(int T, int level) {
  return level == 0 ? T : ((T >> level) > 1 ? (T >> level) : 1);
}

// Walks the work items of one i block whose candidates are c0 .. c0+nc-1:
// emit(level, k, first, n) for the k-th item of each level, levels in order,
// items covering the candidates once, in order.
template <class Emit>
BNB_HD inline void work_walk(int c0, int nc, int T, int tailTiles, Emit emit) {
  int tiles[kWorkLevels], items[kWorkLevels];
  const int L = work_split(nc, T, tailTiles, tiles, items);
  int s = c0;
  for (int l = 0; l < L; l++) {
    const int size = work_item_size(T, l), end = s + tiles[l];
    for (int q = s, k = 0; q < end; q += size, k++) emit(l, k, q, end - q < size ? end - q : size);
    s = end;
  }
}

}  // namespace bnb
