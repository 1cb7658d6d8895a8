// Driver for the transcript hasher test: reads operations from stdin and prints the
// digests of the library's incremental Blake3 (csrc/blake3.cuh, host build).
//   B <n> <hex>        absorb n bytes
//   W <n> <w0> ...     absorb n little-endian words (hex)
//   F                  print finalize()
//   S <n> <w0> ...     print the digest of the state extended by n words twice: from a
//                      snapshot that absorbs them and is finalized, and from
//                      finalize_suffix (no snapshot); state unchanged
#include <cstdio>
#include <vector>

#include "blake3.cuh"

int main() {
  zs::Hasher h;
  char op;
  while (std::scanf(" %c", &op) == 1) {
    if (op == 'B') {
      unsigned n;
      std::scanf("%u", &n);
      std::vector<uint8_t> b(n);
      for (unsigned i = 0; i < n; ++i) {
        unsigned v;
        std::scanf("%2x", &v);
        b[i] = (uint8_t)v;
      }
      h.update(b.data(), n);
    } else if (op == 'W' || op == 'S') {
      unsigned n;
      std::scanf("%u", &n);
      std::vector<uint32_t> w(n);
      for (unsigned i = 0; i < n; ++i) std::scanf("%x", &w[i]);
      std::vector<uint8_t> b(4 * n);
      for (unsigned i = 0; i < 4 * n; ++i) b[i] = (uint8_t)(w[i / 4] >> (8 * (i % 4)));
      if (op == 'W') {
        h.update(b.data(), b.size());
      } else {
        zs::Hasher snap;
        snap.snapshot_from(h);
        snap.update(b.data(), b.size());
        uint8_t o[32];
        snap.finalize(o);
        for (int i = 0; i < 32; ++i) std::printf("%02x", o[i]);
        std::printf("\n");
        uint32_t f[8];  // the same digest without a snapshot
        h.finalize_suffix(b.data(), (unsigned)b.size(), f);
        for (int i = 0; i < 8; ++i)
          for (int k = 0; k < 4; ++k) std::printf("%02x", (f[i] >> (8 * k)) & 0xff);
        std::printf("\n");
      }
    } else if (op == 'F') {
      uint8_t o[32];
      h.finalize(o);
      for (int i = 0; i < 32; ++i) std::printf("%02x", o[i]);
      std::printf("\n");
    }
  }
  return 0;
}
