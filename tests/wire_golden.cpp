// Driver for the golden wire layout test: encodes the struct of
// src/core/serialization.zig:220-250 with the library's wire writer (csrc/host.cuh,
// host build; the writer every proof is serialized with) and prints it as hex.
#include <cstdio>

#include "host.cuh"

int main() {
  zs::WireWriter w;
  const char name[3] = {'a', 'b', 'c'};
  w.bytes(name, 3);
  w.uint_le(0x01020304u, 4);
  const uint16_t rows[2] = {0x0102, 0x0304};
  w.u64(2);
  for (uint16_t r : rows) w.uint_le(r, 2);
  w.flag(true);
  const uint8_t maybe[2] = {0xde, 0xad};
  w.flag(true);
  w.bytes(maybe, 2);
  for (uint8_t b : w.out) std::printf("%02x", b);
  std::printf("\n");
  return 0;
}
