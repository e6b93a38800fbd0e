// Driver around the reference's own CUDA sources (compiled where they lie,
// -I<reference>/include; nothing is copied). TEST INFRASTRUCTURE ONLY: it
// produces the reference's NodeData state after load / insert / delete for
// the golden fixtures, and times the reference's walk and update paths on the
// same GPU as the CUDA path.
//
// The reference is used unmodified; three compile-time redirections in this
// file (not in the reference) make it runnable on a one-GPU box and make its
// host-side behaviour defined:
//   * cudaSetDevice(x) -> cudaSetDevice(0): the reference selects device
//     (g+2)%4, i.e. device 2 (include/gpuMem.cuh:21, include/operation.cuh:66).
//   * sort(...) -> std::stable_sort(...): deleteE's std::sort
//     (include/operation.cuh:218) leaves the order of deletes within one
//     vertex unspecified; stable order makes the swap-remove sequence defined.
//   * global operator new[] returns zero-filled memory (ref_zero_new.cpp,
//     linked in): build() reads the arrays MXLOG and groupNum without
//     initialising them (include/operation.cuh:46-47, :57-58 memset only
//     sizeof(pointer) bytes).
//
// Input (little-endian binary): "BREF" u32 version=1, u32 n, u64 m, f32 rate,
// u32 node2vec, m x (u32 u, u32 v, u32 w) with 0-based ids, then ops:
//   1 INSERT  u64 k, k x (u32 u, u32 v, u32 w)
//   2 DELETE  u64 k, k x (u32 u, u32 slot)
//   3 DUMP    (appends the full NodeData state to the dump file)
//   4 WALK    u32 app (0 deepwalk, 1 node2vec, 2 ppr), u32 reps, u64 seed
//   0 END
// Usage: ref_harness <input> <dump-out|-> ; one JSON line per op on stdout.
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <math.h>
#include <stdlib.h>

#define cudaSetDevice(dev) cudaSetDevice(0)
#define sort(first, last, cmp) std::stable_sort(first, last, cmp)
#include "operation.cuh"
#undef sort
#undef cudaSetDevice

namespace {

struct Reader {
  FILE* f;
  template <class T>
  T get() {
    T v;
    if (fread(&v, sizeof(T), 1, f) != 1) {
      fprintf(stderr, "ref_harness: truncated input\n");
      exit(2);
    }
    return v;
  }
};

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    fprintf(stderr, "ref_harness: %s: %s\n", what, cudaGetErrorString(e));
    exit(3);
  }
}

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <class T>
void put_array(FILE* f, const std::vector<T>& v) {
  uint64_t k = v.size();
  fwrite(&k, 8, 1, f);
  if (k) fwrite(v.data(), sizeof(T), k, f);
}

// D2H of every vertex record and the arrays it points to, written in the
// layout the CPU restatement dumps (0-based ids).
void dump_state(FILE* f, NodeData* ndD, int n) {
  std::vector<NodeData> h(n + 1);
  check(cudaMemcpy(h.data(), ndD, sizeof(NodeData) * (n + 1), cudaMemcpyDeviceToHost), "dump records");
  std::vector<int32_t> logt(n), bits(n), sz(n);
  std::vector<uint32_t> ecnt(n), asz(n), ev, gsz, members;
  std::vector<float> ew, num, ap;
  std::vector<int8_t> grouptp, aa, ab;
  std::vector<int32_t> midx;
  for (int u = 0; u < n; ++u) {
    const NodeData& N = h[u + 1];
    logt[u] = N.LOGT, bits[u] = N.BITS, sz[u] = N.SZ, ecnt[u] = N.edgeSZ, asz[u] = N.aliasTableSZ;
    if (N.edgeSZ) {
      std::vector<NodeData::Edge> e(N.edgeSZ);
      check(cudaMemcpy(e.data(), N.edge, sizeof(NodeData::Edge) * N.edgeSZ, cudaMemcpyDeviceToHost), "edges");
      for (auto& x : e) ev.push_back((uint32_t)(x.v - 1)), ew.push_back(x.weight);
    }
    if (N.LOGT > 0) {
      std::vector<char> tp(N.LOGT);
      std::vector<float> nm(N.LOGT);
      check(cudaMemcpy(tp.data(), N.groupTP, N.LOGT, cudaMemcpyDeviceToHost), "groupTP");
      check(cudaMemcpy(nm.data(), N.num, sizeof(float) * N.LOGT, cudaMemcpyDeviceToHost), "num");
      for (int j = 0; j < N.LOGT; ++j) grouptp.push_back((int8_t)tp[j]), num.push_back(nm[j]);
    }
    if (N.BITS > 0) {
      std::vector<int> gs(N.BITS), grp((size_t)N.BITS * N.SZ), idx((size_t)N.BITS * N.SZ);
      check(cudaMemcpy(gs.data(), N.groupSZ, sizeof(int) * N.BITS, cudaMemcpyDeviceToHost), "groupSZ");
      check(cudaMemcpy(grp.data(), N.group, sizeof(int) * grp.size(), cudaMemcpyDeviceToHost), "group");
      check(cudaMemcpy(idx.data(), N.idx, sizeof(int) * idx.size(), cudaMemcpyDeviceToHost), "idx");
      for (int g = 0; g < N.BITS; ++g) {
        gsz.push_back((uint32_t)gs[g]);
        for (int p = 0; p < gs[g]; ++p) {
          const int slot = grp[(size_t)g * N.SZ + p];
          members.push_back((uint32_t)slot);
          midx.push_back(idx[(size_t)g * N.SZ + slot]);
        }
      }
    }
    if (N.aliasTableSZ) {
      std::vector<NodeData::AliasElement> a(N.aliasTableSZ);
      check(cudaMemcpy(a.data(), N.aliasTable, sizeof(NodeData::AliasElement) * N.aliasTableSZ,
                       cudaMemcpyDeviceToHost),
            "alias");
      for (auto& x : a) ap.push_back(x.p), aa.push_back((int8_t)x.a), ab.push_back((int8_t)x.b);
    }
  }
  fwrite("DUMP", 1, 4, f);
  uint32_t nn = (uint32_t)n;
  fwrite(&nn, 4, 1, f);
  put_array(f, logt), put_array(f, bits), put_array(f, sz), put_array(f, ecnt), put_array(f, asz);
  put_array(f, ev), put_array(f, ew), put_array(f, grouptp), put_array(f, num), put_array(f, gsz);
  put_array(f, members), put_array(f, midx), put_array(f, ap), put_array(f, aa), put_array(f, ab);
  fflush(f);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: ref_harness <input> <dump-out|->\n");
    return 1;
  }
  FILE* in = fopen(argv[1], "rb");
  if (!in) {
    perror("input");
    return 1;
  }
  FILE* out = strcmp(argv[2], "-") ? fopen(argv[2], "wb") : nullptr;
  Reader R{in};
  char magic[4];
  if (fread(magic, 1, 4, in) != 4 || memcmp(magic, "BREF", 4)) {
    fprintf(stderr, "bad magic\n");
    return 1;
  }
  R.get<uint32_t>();
  const int n = (int)R.get<uint32_t>();
  const uint64_t m = R.get<uint64_t>();
  RATE = R.get<float>();
  NODE2VEC = R.get<uint32_t>() != 0;

  mp.init();
  std::vector<int> d(n + 1, 0);
  Edges* edges = new Edges[m];
  for (uint64_t i = 0; i < m; ++i) {
    uint32_t u = R.get<uint32_t>(), v = R.get<uint32_t>(), w = R.get<uint32_t>();
    edges[i] = Edges{(int)u + 1, (int)v + 1, (float)w};
    ++d[u + 1];
  }
  NodeData *nd[GPUS], *ndD[GPUS];
  int* sizeManager = nullptr;
  double t0 = now();
  build(edges, (int)m, nd, ndD, d.data(), &sizeManager, n);
  check(cudaDeviceSynchronize(), "build");
  printf("{\"op\": \"load\", \"n\": %d, \"m\": %llu, \"wall_s\": %.6f}\n", n, (unsigned long long)m, now() - t0);
  delete[] edges;

  int* rwD = nullptr;
  for (;;) {
    const uint32_t op = R.get<uint32_t>();
    if (op == 0) break;
    if (op == 1) {
      const uint64_t k = R.get<uint64_t>();
      Edges* e = new Edges[k];
      for (uint64_t i = 0; i < k; ++i) {
        uint32_t u = R.get<uint32_t>(), v = R.get<uint32_t>(), w = R.get<uint32_t>();
        e[i] = Edges{(int)u + 1, (int)v + 1, (float)w};
        ++d[u + 1];
      }
      t0 = now();
      insert(e, (int)k, nd, ndD, d.data(), sizeManager);
      check(cudaDeviceSynchronize(), "insert");
      printf("{\"op\": \"insert\", \"k\": %llu, \"wall_s\": %.6f}\n", (unsigned long long)k, now() - t0);
      delete[] e;
    } else if (op == 2) {
      const uint64_t k = R.get<uint64_t>();
      Deleted* e = new Deleted[k];
      for (uint64_t i = 0; i < k; ++i) {
        uint32_t u = R.get<uint32_t>(), s = R.get<uint32_t>();
        e[i] = Deleted{(int)u + 1, (int)s};
      }
      t0 = now();
      deleteE(e, (int)k, ndD);
      check(cudaDeviceSynchronize(), "delete");
      printf("{\"op\": \"delete\", \"k\": %llu, \"wall_s\": %.6f}\n", (unsigned long long)k, now() - t0);
      delete[] e;
    } else if (op == 3) {
      if (out) dump_state(out, ndD[0], n);
      printf("{\"op\": \"dump\"}\n");
    } else if (op == 4) {
      const uint32_t app_id = R.get<uint32_t>(), reps = R.get<uint32_t>();
      const uint64_t seed = R.get<uint64_t>();
      const size_t len = (size_t)LEN * (n + 1);
      if (!rwD) check(cudaMalloc((void**)&rwD, len * sizeof(int)), "rwD");
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0), cudaEventCreate(&e1);
      std::vector<int> host(len);
      double steps = 0, ms_total = 0;
      for (uint32_t r = 0; r < reps; ++r) {
        check(cudaMemset(rwD, 0xff, len * sizeof(int)), "memset");
        check(cudaDeviceSynchronize(), "sync");
        cudaEventRecord(e0);
        if (app_id == 0)
          deepwalkKernel<<<BLKSZ, THDSZ>>>(0, 0, n, ndD[0], rwD, 1, seed + r);
        else if (app_id == 1)
          node2vecKernel<<<BLKSZ, THDSZ>>>(0, 0, n, ndD[0], rwD, 1, seed + r);
        else
          pprKernel<<<BLKSZ, THDSZ>>>(0, 0, n, ndD[0], rwD, 1, seed + r);
        cudaEventRecord(e1);
        check(cudaEventSynchronize(e1), "walk");
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        ms_total += ms;
        check(cudaMemcpy(host.data(), rwD, len * sizeof(int), cudaMemcpyDeviceToHost), "walk D2H");
        // produced steps: valid entries after the start, up to the first -1
        for (int w = 0; w < n; ++w) {
          const int* row = host.data() + (size_t)w * LEN;
          for (int j = 1; j < LEN && row[j] != -1; ++j) steps += 1;
        }
      }
      printf("{\"op\": \"walk\", \"app\": %u, \"reps\": %u, \"walks\": %d, \"len\": %d, \"steps\": %.0f, "
             "\"kernel_ms\": %.4f}\n",
             app_id, reps, n, LEN, steps, ms_total);
      cudaEventDestroy(e0), cudaEventDestroy(e1);
    } else {
      fprintf(stderr, "unknown op %u\n", op);
      return 1;
    }
    fflush(stdout);
  }
  if (out) fclose(out);
  fclose(in);
  return 0;
}
