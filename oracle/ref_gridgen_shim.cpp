/*
 * ORACLE PIN — test infrastructure, not product code.
 *
 * The reference's own grid generator (src/gpu/GridGenerator, with the parts of src/basics it
 * uses), compiled for the host from the reference tree where it lies by oracle/Makefile into
 * _ref/libvfref_gridgen.so (real = double). Plain C entry points build a grid with the
 * reference's MultipleGridBuilder -- coarse box, refinement boxes, sphere / cuboid geometries,
 * periodicity, the side boundary conditions of LevelGridBuilder -- and hand out, level by level,
 * the arrays the reference's GridReaderGenerator/GridGenerator.cpp:91-1020 copies into
 * LBMSimulationParameter: node values (coordinates, neighbours, node types), fluid-node
 * indices, the velocity (no-slip included), pressure and geometry BC lists with their q, and the
 * interpolation cells with their offsets. The tests import these arrays with
 * virtualfluids_b200.gridgen and run them against the oracle.
 */
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "gpu/GridGenerator/geometries/Cuboid/Cuboid.h"
#include "gpu/GridGenerator/geometries/Sphere/Sphere.h"
#include "gpu/GridGenerator/grid/BoundaryConditions/Side.h"
#include "gpu/GridGenerator/grid/Grid.h"
#include "gpu/GridGenerator/grid/GridBuilder/MultipleGridBuilder.h"

namespace
{
SideType side_of(int s)
{
    static const SideType sides[] = { SideType::MX, SideType::PX, SideType::MY, SideType::PY,
                                      SideType::MZ, SideType::PZ, SideType::GEOMETRY };
    return sides[s];
}

struct Handle {
    std::shared_ptr<MultipleGridBuilder> builder = std::make_shared<MultipleGridBuilder>();
};

Handle *H(void *h) { return static_cast<Handle *>(h); }

// the 27 q arrays of a list as one block, q27[d * n + i] (Q.q27[d] = block + d * n)
struct QBlock {
    std::vector<real *> ptr;
    QBlock(real *block, size_t n) : ptr(27)
    {
        for (int d = 0; d < 27; ++d)
            ptr[(size_t)d] = block + (size_t)d * n;
    }
};
} // namespace

extern "C" {

int refgg_real_bytes() { return (int)sizeof(real); }

void *refgg_create(double x0, double y0, double z0, double x1, double y1, double z1, double delta)
{
    Handle *h = new Handle();
    h->builder->addCoarseGrid(x0, y0, z0, x1, y1, z1, delta);
    return h;
}

void refgg_destroy(void *h) { delete H(h); }

/* MultipleGridBuilder::addGrid(Cuboid, levelFine) */
void refgg_add_refinement(void *h, double x0, double y0, double z0, double x1, double y1, double z1, int level_fine)
{
    H(h)->builder->addGrid(std::make_shared<Cuboid>(x0, y0, z0, x1, y1, z1), (uint)level_fine);
}

/* MultipleGridBuilder::addGeometry: a solid sphere (kind 0) or cuboid (kind 1) */
void refgg_add_geometry(void *h, int kind, double a, double b, double c, double d, double e, double f)
{
    if (kind == 0)
        H(h)->builder->addGeometry(std::make_shared<Sphere>(a, b, c, d));
    else
        H(h)->builder->addGeometry(std::make_shared<Cuboid>(a, b, c, d, e, f));
}

void refgg_set_periodic(void *h, int px, int py, int pz)
{
    H(h)->builder->setPeriodicBoundaryCondition(px != 0, py != 0, pz != 0);
}

void refgg_build(void *h) { H(h)->builder->buildGrids(false); }

/* side: 0 MX, 1 PX, 2 MY, 3 PY, 4 MZ, 5 PZ, 6 GEOMETRY */
void refgg_set_noslip(void *h, int side) { H(h)->builder->setNoSlipBoundaryCondition(side_of(side)); }
void refgg_set_velocity(void *h, int side, double vx, double vy, double vz)
{
    H(h)->builder->setVelocityBoundaryCondition(side_of(side), vx, vy, vz);
}
void refgg_set_pressure(void *h, int side, double rho) { H(h)->builder->setPressureBoundaryCondition(side_of(side), rho); }

/* GridGenerator.cpp:80 */
void refgg_find_fluid_nodes(void *h) { H(h)->builder->findFluidNodes(false); }

int refgg_levels(void *h) { return (int)H(h)->builder->getNumberOfGridLevels(); }
double refgg_delta(void *h, int level) { return H(h)->builder->getGrid((uint)level)->getDelta(); }

/* numberOfNodes of the level: getNumberOfNodes + 1 (GridGenerator.cpp:100) */
uint32_t refgg_nodes(void *h, int level) { return H(h)->builder->getNumberOfNodes((uint)level) + 1; }

void refgg_node_values(void *h, int level, real *x, real *y, real *z, uint32_t *nbx, uint32_t *nby, uint32_t *nbz,
                       uint32_t *nb_inverse, uint32_t *geo)
{
    H(h)->builder->getNodeValues(x, y, z, nbx, nby, nbz, nb_inverse, geo, level);
}

uint32_t refgg_fluid_count(void *h, int level) { return H(h)->builder->getNumberOfFluidNodes((uint)level); }
void refgg_fluid(void *h, int level, uint32_t *idx) { H(h)->builder->getFluidNodeIndices(idx, level); }

/* velocity BC of the level (every no-slip side is a zero-velocity entry, LevelGridBuilder.cpp:266-285) */
uint32_t refgg_velocity_size(void *h, int level) { return H(h)->builder->getVelocitySize(level); }
void refgg_velocity(void *h, int level, real *vx, real *vy, real *vz, int *k, real *q27)
{
    const uint32_t n = H(h)->builder->getVelocitySize(level);
    H(h)->builder->getVelocityValues(vx, vy, vz, k, level);
    QBlock q(q27, n);
    H(h)->builder->getVelocityQs(q.ptr.data(), level);
}

/* the pressure BCs of the level, one list per side (GridGenerator.cpp:261-300) */
int refgg_pressure_count(void *h, int level) { return (int)H(h)->builder->getNumberOfPressureBoundaryConditions((uint)level); }
uint32_t refgg_pressure_size(void *h, int level, int i)
{
    return (uint32_t)H(h)->builder->getSizeOfPressureBoundaryCondition((uint)level, (uint)i);
}
int refgg_pressure(void *h, int level, int i, real *rho, int *k, int *kN, real *q27)
{
    const uint32_t n = refgg_pressure_size(h, level, i);
    H(h)->builder->getPressureValues(rho, k, kN, (uint)level, (uint)i);
    QBlock q(q27, n);
    H(h)->builder->getPressureQs(q.ptr.data(), (uint)level, (uint)i);
    return (int)H(h)->builder->getPressureBoundaryConditionDirection((uint)level, (uint)i);
}

/* geometry BC of the level (GridGenerator.cpp:923-960). The wall velocities are zero: the no-slip
   geometry BC sets hasGeometryValues, but its velocity lists are filled only by
   fillVelocityLists / setVelocityForPatch, so getGeometryValues would read empty lists here. */
uint32_t refgg_geometry_size(void *h, int level) { return H(h)->builder->getGeometrySize(level); }
void refgg_geometry(void *h, int level, int *k, real *q27, real *vx, real *vy, real *vz)
{
    const uint32_t n = H(h)->builder->getGeometrySize(level);
    H(h)->builder->getGeometryIndices(k, level);
    QBlock q(q27, n);
    H(h)->builder->getGeometryQs(q.ptr.data(), level);
    for (uint32_t i = 0; i < n; ++i)
        vx[i] = vy[i] = vz[i] = 0.0;
}

/* interpolation cells between level and level + 1 (GridGenerator.cpp:993-1020) */
uint32_t refgg_cf_count(void *h, int level) { return H(h)->builder->getNumberOfNodesCF(level); }
uint32_t refgg_fc_count(void *h, int level) { return H(h)->builder->getNumberOfNodesFC(level); }
void refgg_interface(void *h, int level, uint32_t *cf_coarse, uint32_t *cf_fine, uint32_t *fc_coarse, uint32_t *fc_fine,
                     real *cf_x, real *cf_y, real *cf_z, real *fc_x, real *fc_y, real *fc_z)
{
    H(h)->builder->getOffsetCF(cf_x, cf_y, cf_z, level);
    H(h)->builder->getOffsetFC(fc_x, fc_y, fc_z, level);
    H(h)->builder->getGridInterfaceIndices(cf_coarse, cf_fine, fc_coarse, fc_fine, level);
}

} // extern "C"
