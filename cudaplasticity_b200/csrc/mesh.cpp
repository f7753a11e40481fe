// Host mesh of the drop-in API: generators with the reference's node and
// element numbering (so CSR ordering and results match it bit for bit).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cuplast/Mesh.hpp"

namespace cuplast {

namespace {
template <typename T>
T* dup(const T* src, size_t n) {
    T* p = new T[n ? n : 1];
    if (n) std::memcpy(p, src, n * sizeof(T));
    return p;
}
const double kPi = 3.141592653589793;
}  // namespace

void Mesh::clear() {
    delete[] elem3;
    delete[] elem4;
    delete[] elem8;
    delete[] node;
    delete[] secOrdNodes;
    for (int i = 0; i < bordersCount; ++i) delete[] borders[i];
    delete[] borders;
    delete[] borderLength;
    elem3 = elem4 = elem8 = nullptr;
    node = nullptr;
    secOrdNodes = nullptr;
    borders = nullptr;
    borderLength = nullptr;
    bordersCount = 0;
    count3 = count4 = count8 = 0;
    nodeCount = 0;
    analysed = false;
    spaces.clear();
    aspects.clear();
    skewAngles.clear();
    fillPos();
}

Mesh::Mesh(const Mesh& o) { *this = o; }

Mesh& Mesh::operator=(const Mesh& o) {
    if (this == &o) return *this;
    clear();
    useCuda = o.useCuda;
    ramSaved = o.ramSaved;
    count3 = o.count3;
    count4 = o.count4;
    count8 = o.count8;
    nodeCount = o.nodeCount;
    elem3 = dup(o.elem3, 3 * (size_t)count3);
    elem4 = dup(o.elem4, 4 * (size_t)count4);
    elem8 = dup(o.elem8, 8 * (size_t)count8);
    node = dup(o.node, (size_t)nodeCount);
    secOrdNodes = dup(o.secOrdNodes, (size_t)nodeCount);
    bordersCount = o.bordersCount;
    borderLength = dup(o.borderLength, (size_t)bordersCount);
    borders = new int*[bordersCount ? bordersCount : 1];
    for (int b = 0; b < bordersCount; ++b) borders[b] = dup(o.borders[b], (size_t)borderLength[b]);
    analysed = o.analysed;
    spaces = o.spaces;
    aspects = o.aspects;
    skewAngles = o.skewAngles;
    fillPos();
    return *this;
}

Mesh::~Mesh() { clear(); }

void Mesh::assign(int nodes, const double* xy, int c3, const int* e3, int c4, const int* e4,
                  const std::vector<std::vector<int>>& borderLists, int c8, const int* e8) {
    clear();
    nodeCount = nodes;
    node = new vec2[nodes ? nodes : 1];
    secOrdNodes = new bool[nodes ? nodes : 1];
    for (int i = 0; i < nodes; ++i) {
        node[i] = vec2(xy[2 * i], xy[2 * i + 1]);
        secOrdNodes[i] = false;
    }
    count3 = c3;
    count4 = c4;
    elem3 = dup(e3, 3 * (size_t)c3);
    elem4 = dup(e4, 4 * (size_t)c4);
    count8 = e8 ? c8 : 0;
    elem8 = dup(e8, 8 * (size_t)count8);
    for (int e = 0; e < count8; ++e)
        for (int k = 4; k < 8; ++k) {
            const int nd = elem8[8 * (size_t)e + k];
            if (nd >= 0 && nd < nodes) secOrdNodes[nd] = true;
        }
    bordersCount = (int)borderLists.size();
    borderLength = new int[bordersCount ? bordersCount : 1];
    borders = new int*[bordersCount ? bordersCount : 1];
    for (int b = 0; b < bordersCount; ++b) {
        borderLength[b] = (int)borderLists[b].size();
        borders[b] = dup(borderLists[b].data(), borderLists[b].size());
    }
    fillPos();
}

void Mesh::genRectangle(double x1, double x2, double y1, double y2, size_t N1, size_t N2, int order) {
    if (order != 1 && order != 2) throw std::out_of_range("element order must be 1 or 2");
    if (order == 2) {
        N1 *= 2;
        N2 *= 2;
    }
    clear();
    nodeCount = (int)((N1 + 1) * (N2 + 1));
    count4 = (int)(N1 * N2);
    node = new vec2[nodeCount];
    secOrdNodes = new bool[nodeCount];
    std::fill(secOrdNodes, secOrdNodes + nodeCount, false);
    double h1 = (x2 - x1) / N1, h2 = (y2 - y1) / N2;
    for (size_t i = 0; i <= N1; ++i)
        for (size_t j = 0; j <= N2; ++j) node[i * (N2 + 1) + j] = vec2(x1 + h1 * i, y1 + h2 * j);
    elem3 = new int[1];
    elem8 = new int[1];
    elem4 = new int[4 * (size_t)count4];
    for (size_t i = 0; i < N1; ++i)
        for (size_t j = 0; j < N2; ++j) {
            size_t b = 4 * (i * N2 + j);
            elem4[b] = (int)((i + 1) * (N2 + 1) + j + 1);
            elem4[b + 1] = (int)(i * (N2 + 1) + j + 1);
            elem4[b + 2] = (int)(i * (N2 + 1) + j);
            elem4[b + 3] = (int)((i + 1) * (N2 + 1) + j);
        }
    bordersCount = 4;
    borders = new int*[4];
    borderLength = new int[4];
    borderLength[0] = borderLength[2] = (int)N2 + 1;
    borderLength[1] = borderLength[3] = (int)N1 + 1;
    for (int b = 0; b < 4; ++b) borders[b] = new int[borderLength[b]];
    for (size_t i = 0; i <= N2; ++i) {
        borders[0][N2 - i] = (int)((N1 + 1) * (N2 + 1) - i - 1);
        borders[2][N2 - i] = (int)i;
    }
    for (size_t i = 0; i <= N1; ++i) {
        borders[1][N1 - i] = (int)((i + 1) * (N2 + 1) - 1);
        borders[3][N1 - i] = (int)((N1 - i) * (N2 + 1));
    }
    fillPos();
    if (order == 2) remapOrder((int)N2);
}

void Mesh::genRectWithHole(double x1, double x2, double y1, double y2, double holeRad, size_t N1, size_t N2,
                           int order, int radNOverride) {
    if (order != 1 && order != 2) throw std::out_of_range("element order must be 1 or 2");
    clear();
    int borderN = (int)((N1 + N2) * 2);
    int radN = (int)((N1 + N2) / 4);
    radN = (int)std::round(double(radN) * (x2 - x1 + y2 - y1 - 4. * holeRad) * 2. / (x2 - x1 + y2 - y1));
    if (radNOverride > 0) radN = radNOverride;
    if (order == 2) {
        N1 *= 2;
        N2 *= 2;
        borderN *= 2;
        radN *= 2;
    }
    nodeCount = borderN * (radN + 1);
    node = new vec2[nodeCount];
    secOrdNodes = new bool[nodeCount];
    std::fill(secOrdNodes, secOrdNodes + nodeCount, false);
    bordersCount = 5;
    borders = new int*[5];
    borderLength = new int[5];
    borderLength[0] = borderLength[2] = (int)N1 + 1;
    borderLength[1] = borderLength[3] = (int)N2 + 1;
    borderLength[4] = borderN + 1;
    for (int b = 0; b < 5; ++b) borders[b] = new int[borderLength[b]];
    int nodeId = 0;
    double hx = (x2 - x1) / N1, hy = (y2 - y1) / N2;
    for (size_t i = 0; i < N1; ++i, ++nodeId) {
        node[nodeId] = vec2(x1 + i * hx, y1);
        borders[0][i] = nodeId;
    }
    borders[0][borderLength[0] - 1] = nodeId;
    for (size_t j = 0; j < N2; ++j, ++nodeId) {
        node[nodeId] = vec2(x2, y1 + j * hy);
        borders[1][j] = nodeId;
    }
    borders[1][borderLength[1] - 1] = nodeId;
    for (size_t i = 0; i < N1; ++i, ++nodeId) {
        node[nodeId] = vec2(x2 - i * hx, y2);
        borders[2][i] = nodeId;
    }
    borders[2][borderLength[2] - 1] = nodeId;
    for (size_t j = 0; j < N2; ++j, ++nodeId) {
        node[nodeId] = vec2(x1, y2 - j * hy);
        borders[3][j] = nodeId;
    }
    borders[3][borderLength[3] - 1] = 0;
    double phi = 2. * kPi / borderN;
    nodeId = radN * borderN;
    vec2 center(0.5 * (x1 + x2), 0.5 * (y1 + y2));
    double start = phi * (N1 + N2 * 1.5);
    for (int i = 0; i < borderN; ++i, ++nodeId) {
        node[nodeId] = center + vec2(std::cos(start + i * phi), std::sin(start + i * phi)) * holeRad;
        borders[4][borderN - i - 1] = nodeId;
    }
    borders[4][borderLength[4] - 1] = nodeCount - 1;
    vec2 rh = (node[radN * borderN] - node[0]) / radN;
    for (int i = 1; i < radN; ++i) node[i * borderN] = node[0] + rh * i;
    rh = (node[nodeCount - 1] - node[borderN - 1]) / radN;
    for (int i = 1; i < radN; ++i) node[i * borderN + borderN - 1] = node[borderN - 1] + rh * i;
    for (int j = 1; j < borderN; ++j) {
        vec2 r2 = (node[radN * borderN + j] - node[j]) / radN;
        for (int i = 1; i < radN; ++i) node[i * borderN + j] = node[j] + r2 * i;
    }
    count4 = borderN * radN;
    elem3 = new int[1];
    elem8 = new int[1];
    elem4 = new int[4 * (size_t)count4];
    for (int i = 0; i < radN; ++i)
        for (int j = 0; j < borderN - 1; ++j) {
            size_t b = 4 * ((size_t)j * radN + i);
            elem4[b + 1] = (i + 1) * borderN + j;
            elem4[b + 2] = i * borderN + j;
            elem4[b + 3] = i * borderN + j + 1;
            elem4[b + 0] = (i + 1) * borderN + j + 1;
        }
    for (int i = 0; i < radN; ++i) {
        size_t b = 4 * ((size_t)(borderN - 1) * radN + i);
        elem4[b + 1] = (i + 1) * borderN + borderN - 1;
        elem4[b + 2] = i * borderN + borderN - 1;
        elem4[b + 3] = i * borderN;
        elem4[b + 0] = (i + 1) * borderN;
    }
    fillPos();
    renumerateRing(borderN);
    if (order == 2) remapOrder(radN);
}

void Mesh::genRing(double a, double b, size_t N_phi, size_t N_r, int order) {
    if (order != 1 && order != 2) throw std::out_of_range("element order must be 1 or 2");
    if (order == 2) {
        N_phi *= 2;
        N_r *= 2;
    }
    clear();
    nodeCount = (int)((N_r + 1) * N_phi);
    node = new vec2[nodeCount];
    secOrdNodes = new bool[nodeCount];
    std::fill(secOrdNodes, secOrdNodes + nodeCount, false);
    bordersCount = 2;
    borders = new int*[2];
    borderLength = new int[2];
    borderLength[0] = borderLength[1] = (int)N_phi + 1;
    for (int k = 0; k < 2; ++k) borders[k] = new int[borderLength[k]];
    double h_r = (b - a) / N_r, h_phi = 2. * kPi / N_phi;
    for (size_t j = 0; j < N_phi; ++j) {
        for (size_t i = 0; i <= N_r; ++i) {
            double r = b - h_r * i, ph = h_phi * j;
            node[i * N_phi + j] = vec2(r * std::cos(ph), r * std::sin(ph));
        }
        borders[1][N_phi - j] = (int)j;
        borders[0][j] = (int)(N_r * N_phi + j);
    }
    borders[1][0] = 0;
    borders[0][borderLength[1] - 1] = (int)(N_r * N_phi);
    count4 = (int)(N_r * N_phi);
    elem3 = new int[1];
    elem8 = new int[1];
    elem4 = new int[4 * (size_t)count4];
    for (size_t i = 0; i < N_r; ++i)
        for (size_t j = 0; j + 1 < N_phi; ++j) {
            size_t k = 4 * (j * N_r + i);
            elem4[k] = (int)((i + 1) * N_phi + j + 1);
            elem4[k + 3] = (int)(i * N_phi + j + 1);
            elem4[k + 2] = (int)(i * N_phi + j);
            elem4[k + 1] = (int)((i + 1) * N_phi + j);
        }
    for (size_t i = 0; i < N_r; ++i) {
        size_t k = 4 * ((N_phi - 1) * N_r + i);
        elem4[k] = (int)((i + 1) * N_phi);
        elem4[k + 3] = (int)(i * N_phi);
        elem4[k + 2] = (int)(i * N_phi + N_phi - 1);
        elem4[k + 1] = (int)((i + 1) * N_phi + N_phi - 1);
    }
    fillPos();
    renumerateRing((int)N_phi);
    if (order == 2) remapOrder((int)N_r);
}

// Mesh::remapOrder (src/Mesh.cu:443-505): the quads form rows of `width`;
// every 2 x 2 block of them (rows i, i+1 and columns j, j+1, i and j even)
// becomes one 8-node element -- corners from the block's outer corners,
// mid-side nodes from the middles of its outer edges -- the node at the
// block's centre disappears and the remaining nodes keep their order.
void Mesh::remapOrder(int width) {
    count8 = count4 / 4;
    delete[] elem8;
    elem8 = new int[8 * (size_t)count8 + 1];
    std::vector<char> keep(nodeCount, 1);
    const int rows = count4 / width;
    auto q = [&](int i, int j, int k) { return elem4[4 * ((size_t)i * width + j) + k]; };
    for (int i = 0; i < rows; i += 2)
        for (int j = 0; j < width; j += 2) {
            int* e = elem8 + 8 * ((size_t)i * width / 4 + j / 2);
            e[0] = q(i + 1, j + 1, 0);
            e[1] = q(i, j + 1, 1);
            e[2] = q(i, j, 2);
            e[3] = q(i + 1, j, 3);
            e[4] = q(i + 1, j + 1, 1);
            e[5] = q(i, j + 1, 2);
            e[6] = q(i, j, 3);
            e[7] = q(i + 1, j, 0);
            keep[q(i, j, 0)] = 0;
        }
    std::vector<int> renum(nodeCount, -1);
    int kept = 0;
    for (int n = 0; n < nodeCount; ++n)
        if (keep[n]) renum[n] = kept++;
    for (size_t i = 0; i < 8 * (size_t)count8; ++i) elem8[i] = renum[elem8[i]];
    for (int b = 0; b < bordersCount; ++b)
        for (int k = 0; k < borderLength[b]; ++k) borders[b][k] = renum[borders[b][k]];
    vec2* nodes = new vec2[kept ? kept : 1];
    for (int n = 0; n < nodeCount; ++n)
        if (keep[n]) nodes[renum[n]] = node[n];
    delete[] node;
    node = nodes;
    nodeCount = kept;
    delete[] secOrdNodes;
    secOrdNodes = new bool[nodeCount ? nodeCount : 1];
    std::fill(secOrdNodes, secOrdNodes + nodeCount, false);
    for (int e = 0; e < count8; ++e)
        for (int k = 4; k < 8; ++k) secOrdNodes[elem8[8 * e + k]] = true;
    delete[] elem4;
    elem4 = new int[1];
    count4 = 0;
    fillPos();
}

// Mesh::elemSpace8 (src/Mesh.cuh:269-278): the area of the polygon through
// the corners and mid-side nodes, same operation order.
double Mesh::elemSpace8(int e) const {
    double s1 = 0., s2 = 0.;
    for (int i = 8 * e; i < 8 * e + 3; ++i) {
        s1 += node[elem8[i]].x * node[elem8[i + 4]].y + node[elem8[i + 4]].x * node[elem8[i + 1]].y;
        s2 += node[elem8[i]].y * node[elem8[i + 4]].x + node[elem8[i + 4]].y * node[elem8[i + 1]].x;
    }
    s1 += node[elem8[8 * e + 3]].x * node[elem8[8 * e + 7]].y + node[elem8[8 * e + 7]].x * node[elem8[8 * e]].y;
    s2 += node[elem8[8 * e + 3]].y * node[elem8[8 * e + 7]].x + node[elem8[8 * e + 7]].y * node[elem8[8 * e]].x;
    return std::fabs(s1 - s2) * 0.5;
}

void Mesh::renumerateRing(int borderN) {
    // Columns are numbered pairwise from both ends inwards, which keeps the
    // index distance between neighbours small. For an odd column count the
    // reference's last loop writes the old index instead of the new one
    // (src/Mesh.cu:347-349); that is reproduced so the numbering matches it.
    std::vector<int> newNodes(nodeCount, 0);
    int newN = 0, radN = nodeCount / borderN, jBack = borderN - 1, jFront = 0;
    while (jBack > jFront) {
        for (int i = 0; i < radN; ++i) newNodes[i * borderN + jFront] = newN++;
        for (int i = 0; i < radN; ++i) newNodes[i * borderN + jBack] = newN++;
        ++jFront;
        --jBack;
    }
    if (jBack == jFront)
        for (int i = 0; i < radN; ++i) newNodes[newN++] = i * borderN + jFront;
    for (int i = 0; i < 4 * count4; ++i) elem4[i] = newNodes[elem4[i]];
    for (int b = 0; b < bordersCount; ++b)
        for (int j = 0; j < borderLength[b]; ++j) borders[b][j] = newNodes[borders[b][j]];
    std::vector<vec2> nodes(nodeCount);
    for (int i = 0; i < nodeCount; ++i) nodes[newNodes[i]] = node[i];
    std::copy(nodes.begin(), nodes.end(), node);
}

void Mesh::splitToTriangles() {
    int* e3 = new int[6 * (size_t)count4 + 1];
    for (int e = 0; e < count4; ++e) {
        const int* q = elem4 + 4 * (size_t)e;
        int* t = e3 + 6 * (size_t)e;
        t[0] = q[0]; t[1] = q[1]; t[2] = q[2];
        t[3] = q[0]; t[4] = q[2]; t[5] = q[3];
    }
    delete[] elem3;
    elem3 = e3;
    count3 = 2 * count4;
    delete[] elem4;
    elem4 = new int[1];
    count4 = 0;
    fillPos();
}

int Mesh::findMaxIndexDiff() const {
    int mx = 0;
    for (int e = 0; e < count3; ++e)
        for (int i = 3 * e; i < 3 * (e + 1); ++i)
            for (int j = i + 1; j < 3 * (e + 1); ++j) mx = std::max(mx, std::abs(elem3[i] - elem3[j]));
    for (int e = 0; e < count4; ++e)
        for (int i = 4 * e; i < 4 * (e + 1); ++i)
            for (int j = i + 1; j < 4 * (e + 1); ++j) mx = std::max(mx, std::abs(elem4[i] - elem4[j]));
    for (int e = 0; e < count8; ++e)
        for (int i = 8 * e; i < 8 * (e + 1); ++i)
            for (int j = i + 1; j < 8 * (e + 1); ++j) mx = std::max(mx, std::abs(elem8[i] - elem8[j]));
    return mx;
}

double Mesh::elemSpace3(int e) const {
    double s1 = 0., s2 = 0.;
    for (int i = 3 * e + 1; i < 3 * (e + 1); ++i) {
        s1 += node[elem3[i - 1]].x * node[elem3[i]].y;
        s2 += node[elem3[i - 1]].y * node[elem3[i]].x;
    }
    s1 += node[elem3[3 * (e + 1) - 1]].x * node[elem3[3 * e]].y;
    s2 += node[elem3[3 * (e + 1) - 1]].y * node[elem3[3 * e]].x;
    return std::fabs(s1 - s2) * 0.5;
}

double Mesh::elemSpace4(int e) const {
    double s1 = 0., s2 = 0.;
    for (int i = 4 * e + 1; i < 4 * (e + 1); ++i) {
        s1 += node[elem4[i - 1]].x * node[elem4[i]].y;
        s2 += node[elem4[i - 1]].y * node[elem4[i]].x;
    }
    s1 += node[elem4[4 * (e + 1) - 1]].x * node[elem4[4 * e]].y;
    s2 += node[elem4[4 * (e + 1) - 1]].y * node[elem4[4 * e]].x;
    return std::fabs(s1 - s2) * 0.5;
}


// ------------------------------------------------------------ .inp files --
//
// Mesh::loadFromFile (src/Mesh.cu:725-937), same reading rules:
//  * a section starts at a line equal to "*NODE", starting with "*ELEMENT"
//    (blocks of every "TYPE=S3" / "TYPE=S4" / "TYPE=S8R" in it) or equal to
//    "*MPC"; its data lines run up to the first empty line or line starting
//    with '*', and that line is consumed with the block (so a section header
//    right after a block's last data line is not seen);
//  * commas count as blanks; node lines are "id x y ...", element lines
//    "id n1 n2 ..." with 1-based ids; the element id is ignored;
//  * consecutive "*MPC" sections are the borders in order, one line per
//    border node: its first four characters are blanked, the next integer is
//    the node id;
//  * every MPC section brings one reference node in the *NODE list, so the
//    mesh has (node lines - MPC sections) nodes and node lines with a larger
//    id are dropped.
// Quadratic (S8R) elements are read into elem8, and their mid-side nodes
// (local 4..7) marked as second-order nodes.
namespace {

bool is_data(const std::string& l) { return !l.empty() && l[0] != '*'; }

std::string blank_commas(std::string l) {
    for (char& c : l)
        if (c == ',') c = ' ';
    return l;
}

}  // namespace

bool Mesh::loadFromFile(const std::string& fileName) {
    if (fileName.size() < 4 || fileName.substr(fileName.size() - 4) != ".inp")
        throw std::out_of_range("unknown mesh file format (expected .inp)");
    std::ifstream file(fileName);
    if (!file) throw std::out_of_range("there is no such file: " + fileName);
    std::vector<std::string> lines;
    for (std::string l; std::getline(file, l);) lines.push_back(l);

    std::vector<std::pair<int, vec2>> nodeLines;
    std::vector<int> e3, e4, e8;
    std::vector<std::vector<int>> borderLists;
    size_t at = 0;
    auto next = [&](std::string& l) {
        if (at >= lines.size()) return false;
        l = lines[at++];
        return true;
    };
    // reads one data block; returns with `line` holding the consumed terminator
    auto block = [&](std::string& line, auto&& onData) {
        while (next(line)) {
            if (!is_data(line)) return;
            onData(line);
        }
        line.clear();
    };
    std::string line;
    while (next(line)) {
        if (line == "*NODE") {
            block(line, [&](const std::string& l) {
                std::istringstream ss(blank_commas(l));
                int id = 0;
                vec2 p;
                ss >> id >> p.x >> p.y;
                nodeLines.push_back({id - 1, p});
            });
        } else if (line.compare(0, 8, "*ELEMENT") == 0) {
            // the scan goes on over the terminator of each block it reads
            for (size_t i = 0; i < line.length(); ++i) {
                if (line.compare(i, 5, "TYPE=") != 0) continue;
                i += 5;
                const bool t3 = line.compare(i, 2, "S3") == 0, t4 = line.compare(i, 2, "S4") == 0;
                const bool t8 = line.compare(i, 3, "S8R") == 0;
                if (!(t3 || t4 || t8)) continue;
                const int nn = t3 ? 3 : (t4 ? 4 : 8);
                std::vector<int>& dst = t3 ? e3 : (t4 ? e4 : e8);
                block(line, [&](const std::string& l) {
                    std::istringstream ss(blank_commas(l));
                    int id = 0;
                    ss >> id;
                    for (int k = 0; k < nn; ++k) {
                        int v = 0;
                        ss >> v;
                        dst.push_back(v - 1);
                    }
                });
            }
        } else if (line == "*MPC") {
            for (;;) {
                std::vector<int> b;
                block(line, [&](const std::string& l) {
                    std::string t = blank_commas(l);
                    for (size_t k = 0; k < 4 && k < t.size(); ++k) t[k] = ' ';
                    std::istringstream ss(t);
                    int v = 0;
                    ss >> v;
                    b.push_back(v - 1);
                });
                borderLists.push_back(b);
                if (line != "*MPC") break;
            }
        }
    }
    const int nodes = (int)nodeLines.size() - (int)borderLists.size();
    if (nodes <= 0) throw std::out_of_range("mesh file has no nodes");
    std::vector<double> xy(2 * (size_t)nodes, 0.0);
    for (const auto& nl : nodeLines)
        if (nl.first >= 0 && nl.first < nodes) {
            xy[2 * (size_t)nl.first] = nl.second.x;
            xy[2 * (size_t)nl.first + 1] = nl.second.y;
        }
    for (const std::vector<int>* ev : {&e3, &e4, &e8})
        for (int v : *ev)
            if (v < 0 || v >= nodes) throw std::out_of_range("element references a node that does not exist");
    assign(nodes, xy.data(), (int)(e3.size() / 3), e3.data(), (int)(e4.size() / 4), e4.data(), borderLists);
    if (!e8.empty()) {
        count8 = (int)(e8.size() / 8);
        delete[] elem8;
        elem8 = dup(e8.data(), e8.size());
        for (int e = 0; e < count8; ++e)
            for (int k = 4; k < 8; ++k) secOrdNodes[elem8[8 * e + k]] = true;
        fillPos();
    }
    return true;
}

}  // namespace cuplast

// ------------------------------------------------------------ mesh tooling --

namespace cuplast {

namespace {

// Top-down merge sort of keys with their node indices, the order
// renumByDirection numbers the nodes in (src/Mesh.cu:505-535): the halves are
// split at n / 2 and merged taking the left key only when it is strictly
// smaller, so equal keys come out right half first. Kept so that the new
// numbering is the reference's, ties included.
void merge_sort(double* key, int* idx, size_t n, double* kbuf, int* ibuf) {
    if (n < 2) return;
    const size_t half = n / 2;
    merge_sort(key, idx, half, kbuf, ibuf);
    merge_sort(key + half, idx + half, n - half, kbuf + half, ibuf + half);
    size_t a = 0, b = half, o = 0;
    while (a < half && b < n) {
        if (key[a] < key[b]) {
            kbuf[o] = key[a];
            ibuf[o++] = idx[a++];
        } else {
            kbuf[o] = key[b];
            ibuf[o++] = idx[b++];
        }
    }
    while (a < half) {
        kbuf[o] = key[a];
        ibuf[o++] = idx[a++];
    }
    while (b < n) {
        kbuf[o] = key[b];
        ibuf[o++] = idx[b++];
    }
    std::memcpy(key, kbuf, n * sizeof(double));
    std::memcpy(idx, ibuf, n * sizeof(int));
}

}  // namespace

void Mesh::renumByDirection(vec2 direction) {
    const size_t n = (size_t)nodeCount;
    std::vector<double> key(n), kbuf(n);
    std::vector<int> old(n), ibuf(n), now(n);
    for (size_t i = 0; i < n; ++i) {
        old[i] = (int)i;
        key[i] = node[i] * direction;
    }
    merge_sort(key.data(), old.data(), n, kbuf.data(), ibuf.data());
    for (size_t i = 0; i < n; ++i) now[old[i]] = (int)i;
    // the reference leaves elem3 alone (its generators make no triangles);
    // here triangles follow too
    for (size_t i = 0; i < 3 * (size_t)count3; ++i) elem3[i] = now[elem3[i]];
    for (size_t i = 0; i < 4 * (size_t)count4; ++i) elem4[i] = now[elem4[i]];
    for (size_t i = 0; i < 8 * (size_t)count8; ++i) elem8[i] = now[elem8[i]];
    for (int b = 0; b < bordersCount; ++b)
        for (int j = 0; j < borderLength[b]; ++j) borders[b][j] = now[borders[b][j]];
    std::vector<vec2> moved(n);
    for (size_t i = 0; i < n; ++i) moved[now[i]] = node[i];
    std::copy(moved.begin(), moved.end(), node);
    for (size_t i = 0; i < n; ++i) secOrdNodes[i] = false;
    for (int e = 0; e < count8; ++e)
        for (int k = 4; k < 8; ++k) secOrdNodes[elem8[8 * (size_t)e + k]] = true;
    analysed = false;
}

void Mesh::smoothRing(int borderN) {
    const int radN = nodeCount / borderN;
    for (int i = radN - 2; i > 0; --i)
        for (int j = 1; j < borderN - 1; ++j) {
            const vec2 outer = node[(i + 1) * borderN + j];
            node[i * borderN + j] = outer - (outer - node[i * borderN + j]).normalize() * 2. * kPi * outer.norm() / borderN;
        }
}

double Mesh::aspectRatio(int e) const {
    const int b = 4 * e;
    double minSide = (node[elem4[b]] - node[elem4[b + 1]]).norm(), maxSide = minSide;
    for (int i = 0; i < 4; ++i) {
        const double len = (node[elem4[b + (i + 1) % 4]] - node[elem4[b + i]]).norm();
        if (len < minSide) minSide = len;
        else if (len > maxSide) maxSide = len;
    }
    return maxSide / minSide;
}

double Mesh::skewAngleSin(int e) const {
    const int b = 4 * e;
    const vec2 v1 = (node[elem4[b]] + node[elem4[b + 1]] - node[elem4[b + 2]] - node[elem4[b + 3]]) * 0.5;
    const vec2 v2 = (node[elem4[b + 1]] + node[elem4[b + 2]] - node[elem4[b + 3]] - node[elem4[b]]) * 0.5;
    const double dot = v1 * v2;
    return 1. - dot * dot / ((v1.x * v1.x + v1.y * v1.y) * (v2.x * v2.x + v2.y * v2.y));
}

double Mesh::avrElemSize() const {
    double s = 0.;
    for (int e = 0; e < count3; ++e) s += elemSpace3(e);
    for (int e = 0; e < count4; ++e) s += elemSpace4(e);
    for (int e = 0; e < count8; ++e) s += elemSpace8(e);
    return s / elemCount();
}

void Mesh::printAnalysis() {
    spaces.assign(count4, 0.);
    aspects.assign(count4, 0.);
    skewAngles.assign(count4, 0.);
    double avrSpace = 0., minSpace = 1e300, maxSpace = 0., avrAspect = 0., minAspect = 1e300, maxAspect = 0.,
           avrSkew = 0., minSkew = 1e300, maxSkew = 0.;
    for (int e = 0; e < count4; ++e) {
        const double space = elemSpace4(e), aspect = aspectRatio(e), skew = skewAngleSin(e);
        spaces[e] = space;
        aspects[e] = aspect;
        skewAngles[e] = std::acos(skew);
        avrSpace += space;
        avrAspect += aspect;
        avrSkew += skew;
        maxSpace = std::max(maxSpace, space);
        minSpace = std::min(minSpace, space);
        maxAspect = std::max(maxAspect, aspect);
        minAspect = std::min(minAspect, aspect);
        maxSkew = std::max(maxSkew, skew);
        minSkew = std::min(minSkew, skew);
    }
    avrAspect /= count4;
    avrSpace /= count4;
    avrSkew /= count4;
    std::cout << "Mesh analysis:"
              << "\nNodes max index difference in element: " << findMaxIndexDiff() << "\nSpace: avr = " << avrSpace
              << ", min = " << minSpace << ", max = " << maxSpace << "\nAspect ratio " << 100. / avrAspect
              << "%: avr = " << avrAspect << ", min = " << minAspect << ", max = " << maxAspect << "\nSkew angle sin "
              << 100 * avrSkew << "%: avr = " << avrSkew << ", min = " << minSkew << ", max = " << maxSkew << "\n"
              << std::endl;
    analysed = true;
}

void Mesh::saveAsVtk(const std::string& fileName) const {
    std::ofstream f(fileName);
    f << "# vtk DataFile Version 2.0\nMesh\nASCII\nDATASET POLYDATA\n";
    f << "POINTS " << nodeCount << " float\n";
    for (int i = 0; i < nodeCount; ++i) f << node[i].x << " " << node[i].y << " " << 0 << "\n";
    f << "POLYGONS " << elemCount() << " " << 4 * count3 + 5 * count4 + 9 * count8;
    for (int i = 0; i < count3; ++i) {
        f << "\n3 ";
        for (int j = 3 * i; j < 3 * (i + 1); ++j) f << elem3[j] << " ";
    }
    for (int i = 0; i < count4; ++i) {
        f << "\n4 ";
        for (int j = 4 * i; j < 4 * (i + 1); ++j) f << elem4[j] << " ";
    }
    for (int i = 0; i < count8; ++i) {
        f << "\n8 ";
        for (int j = 8 * i; j < 8 * i + 4; ++j) f << elem8[j] << " " << elem8[j + 4] << " ";
    }
    f << "\nCELL_DATA " << elemCount() << "\nSCALARS ElementID int 1\nLOOKUP_TABLE default\n";
    for (int i = 0; i < elemCount(); ++i) f << i << "\n";
    if (analysed) {
        const std::pair<const char*, const std::vector<double>*> q[3] = {
            {"Element_space", &spaces}, {"Element_aspect_ratio", &aspects}, {"Element_skew_angle", &skewAngles}};
        f << "FIELD FieldData 3";
        for (auto& p : q) {
            f << "\n" << p.first << " 1 " << p.second->size() << " float\n";
            for (double v : *p.second) f << v << " ";
        }
    }
    f << "\nPOINT_DATA " << nodeCount << "\nSCALARS NodeID int 1\nLOOKUP_TABLE my_table";
    for (int i = 0; i < nodeCount; ++i) f << "\n" << i;
}

void Mesh::print() const {
    std::cout << "Nodes\n" << nodeCount << "\n";
    for (int i = 0; i < nodeCount; ++i) std::cout << i + 1 << " " << node[i].x << " " << node[i].y << "\n";
    const int counts[3] = {count3, count4, count8}, nen[3] = {3, 4, 8};
    const int* arrays[3] = {elem3, elem4, elem8};
    for (int t = 0; t < 3; ++t) {
        if (!counts[t]) continue;
        std::cout << "\nElements (" << nen[t] << " nodes): " << counts[t] << "\n";
        for (int i = 0; i < counts[t]; ++i) {
            for (int j = nen[t] * i; j < nen[t] * (i + 1); ++j) std::cout << arrays[t][j] + 1 << " ";
            std::cout << "\n";
        }
    }
    std::cout << "\nBorders\n" << bordersCount;
    for (int b = 0; b < bordersCount; ++b) {
        std::cout << "\n" << borderLength[b] << ": ";
        for (int j = 0; j < borderLength[b]; ++j) std::cout << borders[b][j] << " ";
    }
    std::cout << std::endl;
}

}  // namespace cuplast
