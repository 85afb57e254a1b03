// Boundary wiring of the reference's single-level lattice, restated as a table
// (test infrastructure; see oracle_ops.h).  Lattice::setConnectivity
// (Lattice.cpp:500-1394) gives each boundary node a LODI normal direction,
// two normal neighbours (along a diagonal for edge and corner nodes), four
// in-plane neighbours for face nodes, a corner flag and the set of inward
// directions it pushes into.  The table below is indexed by the node's face
// class (fx, fy, fz) in {-1, 0, +1}^3 and was checked against the wiring the
// reference itself builds (tests/golden/topo_*.txt, dumped by
// oracle/ref_build/ref_driver.cpp --topo).
#pragma once

namespace orc {

struct BClass {
    int fx, fy, fz;   // face class
    int normalDir;    // Node::normalDir_ (0:-x 1:-y 2:+x 3:+y 4:-z 5:+z outward normal)
    int n1[3], n2[3]; // offsets of the first and second normal neighbour
    int corner;       // Node::isCorner_ (no transverse terms)
    int push[5];      // pushed directions, -1 terminated
};

// clang-format off
constexpr BClass kBoundaryClasses[26] = {
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

inline const BClass* boundaryClass(int fx, int fy, int fz) {
    for (const BClass& c : kBoundaryClasses)
        if (c.fx == fx && c.fy == fy && c.fz == fz) return &c;
    return nullptr;
}

// In-plane neighbour offsets of face nodes: tangent1 (two), tangent2 (two);
// x before y before z (Lattice.cpp:524-531, 617-624, 855-862).
inline void faceTangents(int fx, int fy, int fz, int t[4][3]) {
    int a1, a2;  // the two in-plane axes
    if (fx != 0) { a1 = 1; a2 = 2; }
    else if (fy != 0) { a1 = 0; a2 = 2; }
    else { (void)fz; a1 = 0; a2 = 1; }
    for (int m = 0; m < 4; ++m) t[m][0] = t[m][1] = t[m][2] = 0;
    t[0][a1] = 1; t[1][a1] = -1; t[2][a2] = 1; t[3][a2] = -1;
}

}  // namespace orc
