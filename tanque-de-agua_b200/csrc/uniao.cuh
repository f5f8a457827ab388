// uniao.cuh — lock-free union-find over int parent arrays (4-connected component labelling of
// the air pockets and of the pressure solve's closed regions).  Linking always puts the larger
// root under the smaller, so a component's root is its smallest index.  Every retry loop is
// bounded by LIMITE_UNIAO; unir returns false when it gives up (the caller raises an error).
#pragma once

namespace tq {

constexpr int LIMITE_UNIAO = 1 << 22;

__device__ inline int raiz(int* pai, int a) {
  for (int g = 0; g < LIMITE_UNIAO; g++) {
    int p = pai[a];
    if (p == a) return a;
    int gp = pai[p];
    if (gp != p) pai[a] = gp;  // path halving: gp is an ancestor of a
    a = p;
  }
  return a;
}
__device__ inline bool unir(int* pai, int a, int b) {
  for (int g = 0; g < LIMITE_UNIAO; g++) {
    a = raiz(pai, a);
    b = raiz(pai, b);
    if (a == b) return true;
    if (a < b) { int t = a; a = b; b = t; }
    if (atomicCAS(&pai[a], a, b) == a) return true;  // larger root under the smaller
  }
  return false;
}
// The root by a read-only walk (for the flattening pass, whose only writes store roots).
__device__ inline int raizLeitura(const int* pai, int a) {
  for (int g = 0; g < LIMITE_UNIAO; g++) {
    int p = pai[a];
    if (p == a) break;
    a = p;
  }
  return a;
}

}  // namespace tq
