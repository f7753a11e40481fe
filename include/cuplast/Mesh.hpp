// Mesh of the drop-in API: the public fields and generators of the
// reference's class Mesh (src/Mesh.cuh:22-318), host side only. The device
// copy lives in the solver instance (cp_instance), so there are no dev_*
// fields and no meshToGPU / meshToRAM round trips.
#pragma once

#include <string>
#include <vector>

#include "vec2.hpp"

namespace cuplast {

class CUPLAST_CXX_API Mesh {
public:
    bool useCuda = true;   // kept for source compatibility; the solver always runs on the GPU
    bool ramSaved = true;

    int count3 = 0, count4 = 0, count8 = 0;
    int* elem3 = nullptr;
    int* elem4 = nullptr;
    int* elem8 = nullptr;
    int elemPos[3] = {};

    int nodeCount = 0;
    vec2* node = nullptr;
    bool* secOrdNodes = nullptr;

    int bordersCount = 0;
    int* borderLength = nullptr;
    int** borders = nullptr;

    // quality of the 4-node elements, filled by printAnalysis (and then
    // written by saveAsVtk)
    bool analysed = false;
    std::vector<double> spaces, aspects, skewAngles;

    Mesh() = default;
    Mesh(const Mesh& other);
    Mesh& operator=(const Mesh& other);
    ~Mesh();

    int elemCount() const { return elemPos[2]; }

    // src/Mesh.cu:17-110
    void genRectangle(double x1, double x2, double y1, double y2, size_t N1, size_t N2, int order = 1);
    // src/Mesh.cu:112-246. radN > 0 overrides the reference's radial count
    // (which it ties to the perimeter count): the O-grid of the benchmarks.
    void genRectWithHole(double x1, double x2, double y1, double y2, double holeRad, size_t N1, size_t N2,
                         int order = 1, int radN = 0);
    // src/Mesh.cu:249-329
    void genRing(double a, double b, size_t N_phi, size_t N_r, int order = 1);
    // src/Mesh.cu:332-380
    void renumerateRing(int borderN);
    // src/Mesh.cu:443-505: quads in rows of `width` -> 8-node elements
    // (what the generators do for order = 2)
    void remapOrder(int width);
    // Extension: every quad (n1,n2,n3,n4) becomes (n1,n2,n3), (n1,n3,n4).
    void splitToTriangles();
    // src/Mesh.cu:417-440
    int findMaxIndexDiff() const;

    double elemSpace3(int e) const;
    double elemSpace4(int e) const;
    double elemSpace8(int e) const;

    // Mesh tooling of the reference (host side):
    // src/Mesh.cu:537-636: renumber the nodes by their projection on a
    // direction (element, border and second-order node arrays follow)
    void renumByDirection(vec2 direction = vec2(1., 1.));
    // src/Mesh.cu:386-416: moves the inner rings of an O-grid with borderN
    // columns so that each cell's radial side matches its ring's arc step
    void smoothRing(int borderN);
    // src/Mesh.cuh:279-317: largest over smallest side, 1 - cos^2 of the
    // angle between the mid-lines (4-node element e), mean element area
    double aspectRatio(int e) const;
    double skewAngleSin(int e) const;
    double avrElemSize() const;
    // src/Mesh.cu:1032-1080: per-element area, aspect ratio and skew angle
    // of the 4-node elements, with a summary on std::cout
    void printAnalysis();
    // src/Mesh.cu:939-990 and 992-1030: the mesh as VTK polygons; the arrays
    // on std::cout
    void saveAsVtk(const std::string& fileName) const;
    void print() const;
    // the reference's host/device copies; the solver instance holds the
    // device copy here, so both do nothing
    void meshToRAM() {}
    void meshToGPU() {}

    // src/Mesh.cu:725-937: a mesh from an .inp file (nodes, S3/S4/S8R
    // element blocks, *MPC border blocks); true when loaded. Throws
    // std::out_of_range on a bad file.
    bool loadFromFile(const std::string& fileName);

    // Replaces the arrays (takes copies). The mid-side nodes of 8-node
    // elements become second-order nodes (secOrdNodes).
    void assign(int nodes, const double* xy, int c3, const int* e3, int c4, const int* e4,
                const std::vector<std::vector<int>>& borderLists, int c8 = 0, const int* e8 = nullptr);

private:
    void clear();
    void fillPos() {
        elemPos[0] = count3;
        elemPos[1] = elemPos[0] + count4;
        elemPos[2] = elemPos[1] + count8;
    }
};

}  // namespace cuplast
