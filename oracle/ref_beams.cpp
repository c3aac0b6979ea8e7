/*
 * Reference harness TU for BB1D (test infrastructure): compiles the
 * reference's Beams/PhBeams.cxx unchanged.  Built twice by
 * oracle/build_ref.py: once as is (USE_GRID, the reference default,
 * PhBeams.hxx:30-34) and once with UPBP_REF_USE_BRUTE (the reference's
 * brute-force AccelStruct, PhBrute.hxx:36-104) under the class names
 * PhotonBeamsEvaluatorBrute / AccelStructBrute.
 */
#include <vector>
#include <list>
#include <forward_list>
#include <string>
#include <sstream>
#include <iostream>
#include <iomanip>
#include <algorithm>
#include <cmath>
#if defined(UPBP_REF_USE_BRUTE)
#define PhotonBeamsEvaluator PhotonBeamsEvaluatorBrute
#define AccelStruct AccelStructBrute
#else
// the grid's cell lists are private members (Grid.hxx:644-646); ref_grid_export reads them
#define private public
#define protected public
#endif
#include "Beams/PhBeams.cxx"

#if !defined(UPBP_REF_USE_BRUTE)
/* The grid of a built evaluator: mCells, mPointers as indices from `base` (the beams array) and
 * mPdfs.  AccelStruct derives privately from Grid<AccelStruct> (PhGrid.hxx:36): a C-style cast
 * reaches the base. */
int ref_grid_export(const PhotonBeamsEvaluator& e, const PhotonBeam* base, uint32_t* cells, int32_t* beams, float* pdfs,
                    int64_t* n_cells, int64_t* n_entries)
{
    if (!e.accelStruct) return -2;
    const Grid<AccelStruct>* g = (const Grid<AccelStruct>*)e.accelStruct;
    if (n_cells) *n_cells = (int64_t)g->mCells.size();
    if (n_entries) *n_entries = (int64_t)g->mPointers.size();
    if (cells) std::copy(g->mCells.begin(), g->mCells.end(), cells);
    if (beams)
        for (size_t i = 0; i < g->mPointers.size(); ++i) beams[i] = (int32_t)(g->mPointers[i] - base);
    if (pdfs) std::copy(g->mPdfs.begin(), g->mPdfs.end(), pdfs);
    return 0;
}
#endif

#if defined(UPBP_REF_USE_BRUTE)
/* Opaque entry points so the main harness TU (which sees the grid class
 * under the reference name) can drive the brute-force evaluator. */
void* ref_brute_create(const Scene& scene, PhotonBeamsArray& beams, float radius, int knn)
{
    PhotonBeamsEvaluatorBrute* e = new PhotonBeamsEvaluatorBrute(scene);
    e->build(beams, knn > 0 ? KNN_RADIUS : CONSTANT_RADIUS, radius, knn, false);
    return e;
}
Rgb ref_brute_eval(void* h, BeamType bt, const Ray& ray, const VolumeSegments& segs, uint tech, uint rsf,
                   embree::AdditionalRayDataForMis* data)
{
    return static_cast<PhotonBeamsEvaluatorBrute*>(h)->evalBeamBeamEstimate(bt, ray, segs, tech, rsf, data, NULL);
}
Rgb ref_brute_eval_lite(void* h, BeamType bt, const Ray& ray, const LiteVolumeSegments& segs, uint tech, uint rsf,
                        embree::AdditionalRayDataForMis* data)
{
    return static_cast<PhotonBeamsEvaluatorBrute*>(h)->evalBeamBeamEstimate(bt, ray, segs, tech, rsf, data, NULL);
}
void ref_brute_destroy(void* h)
{
    PhotonBeamsEvaluatorBrute* e = static_cast<PhotonBeamsEvaluatorBrute*>(h);
    e->destroy();
    delete e;
}
#endif
