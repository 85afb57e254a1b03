// Boundary wiring of a single-level lattice, as the reference builds it in
// Lattice::setConnectivity (Lattice.cpp:500-1394), restated as a table over
// the 26 face classes (fx, fy, fz) of a boundary node: LODI normal direction,
// first and second normal neighbour (along a diagonal for edge and corner
// nodes), the corner flag (no transverse terms) and the inward directions the
// node pushes into (BoundaryNode::transport).  Face nodes also get four
// in-plane neighbours for the transverse LODI terms.  Periodic axes (an
// extension) carry no boundary nodes; offsets along them wrap.
#pragma once

namespace acp {

struct BoundaryClass {
    int fx, fy, fz;
    int normalDir;
    int n1[3], n2[3];
    int corner;
    int push[5];  // -1 terminated
};

// clang-format off
static const BoundaryClass kBoundaryClasses[26] = {
    {-1,-1,-1, 0, { 1, 0, 0}, { 2, 0, 0}, 1, {-1}},
    {-1,-1, 0, 0, { 1, 1, 0}, { 2, 2, 0}, 1, {16, -1}},
    {-1,-1, 1, 0, { 1, 0, 0}, { 2, 0, 0}, 1, {-1}},
    {-1, 0,-1, 0, { 1, 0, 1}, { 2, 0, 2}, 1, {6, -1}},
    {-1, 0, 0, 0, { 1, 0, 0}, { 2, 0, 0}, 0, {0, 6, 7, 15, 16}},
    {-1, 0, 1, 0, { 1, 0,-1}, { 2, 0,-2}, 1, {7, -1}},
    {-1, 1,-1, 0, { 1, 0, 0}, { 2, 0, 0}, 1, {-1}},
    {-1, 1, 0, 0, { 1,-1, 0}, { 2,-2, 0}, 1, {15, -1}},
    {-1, 1, 1, 0, { 1, 0, 0}, { 2, 0, 0}, 1, {-1}},
    { 0,-1,-1, 1, { 0, 1, 1}, { 0, 2, 2}, 1, {8, -1}},
    { 0,-1, 0, 1, { 0, 1, 0}, { 0, 2, 0}, 0, {1, 8, 9, 14, 16}},
    { 0,-1, 1, 1, { 0, 1,-1}, { 0, 2,-2}, 1, {9, -1}},
    { 0, 0,-1, 4, { 0, 0, 1}, { 0, 0, 2}, 0, {4, 6, 8, 10, 12}},
    { 0, 0, 1, 5, { 0, 0,-1}, { 0, 0,-2}, 0, {5, 7, 9, 11, 13}},
    { 0, 1,-1, 3, { 0,-1, 1}, { 0,-2, 2}, 1, {12, -1}},
    { 0, 1, 0, 3, { 0,-1, 0}, { 0,-2, 0}, 0, {3, 12, 13, 15, 17}},
    { 0, 1, 1, 3, { 0,-1,-1}, { 0,-2,-2}, 1, {13, -1}},
    { 1,-1,-1, 4, {-1, 1, 1}, {-2, 2, 2}, 1, {-1}},
    { 1,-1, 0, 1, {-1, 1, 0}, {-2, 2, 0}, 1, {14, -1}},
    { 1,-1, 1, 5, {-1, 1,-1}, {-2, 2,-2}, 1, {-1}},
    { 1, 0,-1, 4, {-1, 0, 1}, {-2, 0, 2}, 1, {10, -1}},
    { 1, 0, 0, 2, {-1, 0, 0}, {-2, 0, 0}, 0, {2, 10, 11, 14, 17}},
    { 1, 0, 1, 5, {-1, 0,-1}, {-2, 0,-2}, 1, {11, -1}},
    { 1, 1,-1, 4, {-1,-1, 1}, {-2,-2, 2}, 1, {-1}},
    { 1, 1, 0, 3, {-1,-1, 0}, {-2,-2, 0}, 1, {17, -1}},
    { 1, 1, 1, 5, {-1,-1,-1}, {-2,-2,-2}, 1, {-1}},
};
// clang-format on

inline int faceCode(int fx, int fy, int fz) { return (fx + 1) * 9 + (fy + 1) * 3 + (fz + 1); }

inline const BoundaryClass* boundaryClass(int fx, int fy, int fz) {
    for (const BoundaryClass& c : kBoundaryClasses)
        if (c.fx == fx && c.fy == fy && c.fz == fz) return &c;
    return nullptr;
}

// in-plane neighbour offsets of a face node: tangent1 (+,-), tangent2 (+,-),
// with x before y before z (Lattice.cpp:524-531, 617-624, 855-862)
inline void faceTangents(int fx, int fy, int fz, int t[4][3]) {
    int a1, a2;
    if (fx != 0) { a1 = 1; a2 = 2; }
    else if (fy != 0) { a1 = 0; a2 = 2; }
    else { (void)fz; a1 = 0; a2 = 1; }
    for (int m = 0; m < 4; ++m) t[m][0] = t[m][1] = t[m][2] = 0;
    t[0][a1] = 1; t[1][a1] = -1; t[2][a2] = 1; t[3][a2] = -1;
}

}  // namespace acp
