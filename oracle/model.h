/*
 * oracle/model.h -- TEST INFRASTRUCTURE (the CPU oracle), not the product.
 *
 * KUKA iiwa14 rigid-body model used by the oracle, written as URDF-style
 * physical parameters.  The reference does not ship these parameters in this
 * form: it ships GRiD-generated precomputed spatial matrices
 * (rbdfiles/iiwa_eepos_grid.cuh:907-1674, q-dependent entries at :1768-1853 and
 * :1857-1913).  The values below are the physical quantities those matrices
 * encode (mass, centre of mass and rotational inertia about the centre of mass
 * of each link; translation and fixed rotation of each joint origin; every
 * joint revolute about its local z axis; gravity 0 as in
 * rbdfiles/iiwa_eepos_plant.cuh:50-51).  They are pinned by the reference's
 * own forward-kinematics golden file (testfiles/0_0_eepos.traj) and by the
 * explicit-Euler consistency of testfiles/0_0_traj.csv.
 */
#ifndef GPT_ORACLE_MODEL_H
#define GPT_ORACLE_MODEL_H

#define ORC_NJ 7

/* joint origin translation in the parent frame (m) */
static const double ORC_JOINT_P[ORC_NJ][3] = {
    {0.0, 0.0, 0.1575}, {0.0, 0.0, 0.2025}, {0.0, 0.2045, 0.0}, {0.0, 0.0, 0.2155},
    {0.0, 0.1845, 0.0}, {0.0, 0.0, 0.2155}, {0.0, 0.081, 0.0}};

/* fixed joint-origin rotation (row-major 3x3, child->parent); kinds:
 * 0 = identity, 1 = rpy(pi/2, 0, pi) == rpy(-pi/2, pi, 0), 2 = rpy(pi/2, 0, 0) */
static const int ORC_JOINT_R_KIND[ORC_NJ] = {0, 1, 1, 2, 1, 2, 1};

static const double ORC_MASS[ORC_NJ] = {5.76, 6.35, 3.5, 3.5, 3.5, 1.8, 1.2};
static const double ORC_COM[ORC_NJ][3] = {
    {0.0, -0.03, 0.12}, {0.0003, 0.059, 0.042}, {0.0, 0.03, 0.13}, {0.0, 0.067, 0.034},
    {0.0001, 0.021, 0.076}, {0.0, 0.0006, 0.0004}, {0.0, 0.0, 0.02}};
/* rotational inertia about the COM: ixx iyy izz ixy ixz iyz (tensor entries) */
static const double ORC_INERTIA[ORC_NJ][6] = {
    {0.121, 0.116, 0.0175, 0.0, 0.0, -0.021},
    {0.0638, 0.0416, 0.0331, 0.0001, 0.00008, 0.0157},
    {0.0873, 0.083, 0.0108, 0.0, 0.0, 0.014},
    {0.0368, 0.02045, 0.02171, 0.0, 0.0, 0.008},
    {0.0318, 0.028916, 0.006, 0.000007, 0.000027, 0.005586},
    {0.0049, 0.0047, 0.0036, 0.0, 0.0, 0.0},
    {0.0055, 0.0055, 0.005, 0.0, 0.0, 0.0}};

#endif
