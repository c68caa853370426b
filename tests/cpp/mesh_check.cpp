// Parses each OBJ file named on the command line through the C ABI's mesh loader
// (eos_mesh_parse_obj / eos_mesh_get_info / eos_mesh_get_data / eos_mesh_destroy) and
// touches every value it returns.  Built with AddressSanitizer and UBSan by
// tests/test_sanitizers.py, which feeds it the mesh fixtures, the reference's models and
// fuzzed inputs; a sanitizer report ends the process with a non-zero status.  Prints one
// line per file: the status and, when it parsed, the vertex and triangle counts.
#include <cstdint>
#include <cstdio>
#include <vector>

#include "eos_c.h"

int main(int argc, char** argv) {
  for (int i = 1; i < argc; ++i) {
    std::FILE* f = std::fopen(argv[i], "rb");
    if (!f) return 2;
    std::vector<char> text;
    char buf[65536];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) text.insert(text.end(), buf, buf + n);
    std::fclose(f);
    eos_mesh* m = nullptr;
    const eos_status st = eos_mesh_parse_obj(text.data(), text.size(), &m);
    if (st != EOS_OK) {
      std::printf("%d\n", (int)st);
      continue;
    }
    eos_mesh_info info{};
    if (eos_mesh_get_info(m, &info) != EOS_OK) return 3;
    std::vector<float> v((size_t)info.n_verts * 3), nrm((size_t)info.n_verts * 3);
    std::vector<uint32_t> t((size_t)info.n_tris * 3);
    if (eos_mesh_get_data(m, v.data(), nrm.data(), t.data()) != EOS_OK) return 4;
    double sum = 0.0;
    for (float x : v) sum += x;
    for (float x : nrm) sum += x;
    for (uint32_t x : t) {
      if (x >= info.n_verts) return 5;  // every index names a vertex
      sum += x;
    }
    eos_mesh_destroy(m);
    std::printf("0 %u %u %g\n", info.n_verts, info.n_tris, sum);
  }
  return 0;
}
