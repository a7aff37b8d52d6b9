// gpt_model.cuh -- KUKA iiwa14 rigid-body model for the device kernels.
//
// The reference evaluates the arm with GRiD-generated code whose model is a
// table of precomputed spatial matrices (rbdfiles/iiwa_eepos_grid.cuh:907-1674,
// q-dependent entries written at :1768-1853 and :1857-1913).  Here the model
// is the underlying URDF-style data -- per link mass, centre of mass and
// rotational inertia about it; per joint the origin translation and a fixed
// rotation; every joint revolute about local z; gravity 0
// (rbdfiles/iiwa_eepos_plant.cuh:50-51) -- and the spatial quantities the
// recursive algorithms need are derived from it at compile time.
#pragma once

namespace gpt {
namespace model {

constexpr int NJ = 7;

// joint origin translation in the parent frame (m)
constexpr float kJointP[NJ][3] = {{0.f, 0.f, 0.1575f}, {0.f, 0.f, 0.2025f}, {0.f, 0.2045f, 0.f},
                                  {0.f, 0.f, 0.2155f}, {0.f, 0.1845f, 0.f}, {0.f, 0.f, 0.2155f},
                                  {0.f, 0.081f, 0.f}};
// fixed joint-origin rotation kind: 0 identity, 1 rpy(pi/2,0,pi), 2 rpy(pi/2,0,0)
constexpr int kJointKind[NJ] = {0, 1, 1, 2, 1, 2, 1};

constexpr double kMass[NJ] = {5.76, 6.35, 3.5, 3.5, 3.5, 1.8, 1.2};
constexpr double kCom[NJ][3] = {{0.0, -0.03, 0.12},     {0.0003, 0.059, 0.042}, {0.0, 0.03, 0.13},
                                {0.0, 0.067, 0.034},    {0.0001, 0.021, 0.076}, {0.0, 0.0006, 0.0004},
                                {0.0, 0.0, 0.02}};
// rotational inertia about the COM: ixx iyy izz ixy ixz iyz
constexpr double kInertia[NJ][6] = {{0.121, 0.116, 0.0175, 0.0, 0.0, -0.021},
                                    {0.0638, 0.0416, 0.0331, 0.0001, 0.00008, 0.0157},
                                    {0.0873, 0.083, 0.0108, 0.0, 0.0, 0.014},
                                    {0.0368, 0.02045, 0.02171, 0.0, 0.0, 0.008},
                                    {0.0318, 0.028916, 0.006, 0.000007, 0.000027, 0.005586},
                                    {0.0049, 0.0047, 0.0036, 0.0, 0.0, 0.0},
                                    {0.0055, 0.0055, 0.005, 0.0, 0.0, 0.0}};

// Rotational inertia about the link origin: Ic + m (|c|^2 I - c c^T), 6 unique
// entries xx yy zz xy xz yz.
constexpr double ibar(int i, int e)
{
    const double m = kMass[i];
    const double cx = kCom[i][0], cy = kCom[i][1], cz = kCom[i][2];
    const double cc = cx * cx + cy * cy + cz * cz;
    switch (e) {
    case 0: return kInertia[i][0] + m * (cc - cx * cx);
    case 1: return kInertia[i][1] + m * (cc - cy * cy);
    case 2: return kInertia[i][2] + m * (cc - cz * cz);
    case 3: return kInertia[i][3] - m * cx * cy;
    case 4: return kInertia[i][4] - m * cx * cz;
    default: return kInertia[i][5] - m * cy * cz;
    }
}

}  // namespace model
}  // namespace gpt
