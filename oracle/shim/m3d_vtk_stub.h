/* oracle/shim/m3d_vtk_stub.h -- TEST INFRASTRUCTURE ONLY (part of the CPU oracle).
 * Minimal stand-ins for the VTK classes named by the reference headers
 * (include/FFT_analysis3D.hpp:12-23, include/FFT_thermal3D.hpp:12-23).  Only
 * vtiWriter (src/3d/FFT_analysis3D.cpp:1056-1104) uses them, as an XML file
 * writer; the oracle never calls vtiWriter, so Write() writes nothing.
 * No rendering class is used by the reference sources. */
#ifndef M3D_VTK_STUB_H
#define M3D_VTK_STUB_H
#include <string>
#include <vector>
#define VTK_MAJOR_VERSION 7
#define VTK_DOUBLE 11
template <class T> class vtkSmartPointer {
public:
    T* p = nullptr;
    static vtkSmartPointer New() { vtkSmartPointer s; s.p = new T(); return s; }
    T* operator->() const { return p; }
};
class vtkImageData {
public:
    int dims[3] = {0, 0, 0};
    int ncomp = 0;
    std::vector<double> buf;
    void SetDimensions(int x, int y, int z) { dims[0] = x; dims[1] = y; dims[2] = z; }
    void AllocateScalars(int, int n) { ncomp = n; buf.assign((size_t)dims[0] * dims[1] * dims[2] * n, 0.0); }
    int* GetDimensions() { return dims; }
    void* GetScalarPointer(int x, int y, int z) {
        return buf.data() + ((size_t)x + (size_t)dims[0] * (y + (size_t)dims[1] * z)) * ncomp;
    }
};
class vtkXMLImageDataWriter {
public:
    std::string name;
    void SetFileName(const char* f) { name = f; }
    void SetInputData(vtkImageData*) {}
    void SetInputData(const vtkSmartPointer<vtkImageData>&) {}
    int Write() { return 1; }
};
#endif
