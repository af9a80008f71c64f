// Tiny array dumper used by the reference harnesses (test infrastructure).
// Each call writes <dir>/<name>.bin (raw little-endian) and appends
// "<name> <dtype> <dim0> <dim1> ..." to <dir>/manifest.txt, which
// tests/golden/make_golden.py reads back with numpy.
#ifndef ROME_ORACLE_DUMP_H
#define ROME_ORACLE_DUMP_H
#include <cstdio>
#include <string>
#include <vector>

class Dumper {
  public:
    explicit Dumper(const std::string& dir) : dir_(dir) {
        std::string m = dir_ + "/manifest.txt";
        manifest_ = std::fopen(m.c_str(), "w");
    }
    ~Dumper() {
        if (manifest_) std::fclose(manifest_);
    }
    template <typename T>
    void put(const std::string& name, const T* data, const std::vector<long>& shape, const char* dtype) {
        long n = 1;
        for (long d : shape) n *= d;
        std::string path = dir_ + "/" + name + ".bin";
        FILE* f = std::fopen(path.c_str(), "wb");
        if (n > 0) std::fwrite(data, sizeof(T), (size_t)n, f);
        std::fclose(f);
        std::fprintf(manifest_, "%s %s", name.c_str(), dtype);
        for (long d : shape) std::fprintf(manifest_, " %ld", d);
        std::fprintf(manifest_, "\n");
        std::fflush(manifest_);
    }
    void f64(const std::string& name, const double* p, std::vector<long> shape) { put(name, p, shape, "f8"); }
    void i32(const std::string& name, const int* p, std::vector<long> shape) { put(name, p, shape, "i4"); }
    void i8(const std::string& name, const char* p, std::vector<long> shape) { put(name, p, shape, "i1"); }
    void scalar(const std::string& name, double v) { f64(name, &v, {1}); }
    void iscalar(const std::string& name, int v) { i32(name, &v, {1}); }

  private:
    std::string dir_;
    FILE* manifest_ = nullptr;
};
#endif
