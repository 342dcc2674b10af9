/* oracle/shim/CImg.h -- TEST INFRASTRUCTURE ONLY (part of the CPU oracle).
 * The reference's 3-D solver headers include <CImg.h> and open its namespace
 * (include/FFT_analysis3D.hpp:7,28) but the 3-D solver sources call nothing in
 * it; this stand-in replaces the vendored image library for the oracle
 * build, which keeps X11 out of it. */
#ifndef M3D_CIMG_STUB_H
#define M3D_CIMG_STUB_H
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <sys/stat.h>
#include <vector>
namespace cimg_library {
/* In-memory image with the members the reconstruction source names
   (constructor from two perpendicular sections, saveRecImages); the oracle
   calls neither path, so nothing is ever loaded or written. */
template <class T>
class CImg {
public:
    CImg() {}
    CImg(int w, int h, int d = 1) : w_(w), h_(h), d_(d), px_((size_t)w * h * d) {}
    int width() const { return w_; }
    int height() const { return h_; }
    T atXY(int x, int y) const { return px_[(size_t)y * w_ + x]; }
    T& operator()(int x, int y, int z) { return px_[((size_t)z * h_ + y) * w_ + x]; }
    const CImg& save(const char*) const { return *this; }
private:
    int w_ = 0, h_ = 0, d_ = 0;
    std::vector<T> px_;
};
}  // namespace cimg_library
#endif
