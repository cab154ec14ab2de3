/*
 * g2o_io.h -- the .g2o text format for the graphs the device path optimizes.
 *
 * Host-only entry points of libg2o_b200.so (no CUDA call, usable without a
 * GPU). They read and write the text that g2o's OptimizableGraph::load / save
 * read and write for the vertex, edge and parameter types of the device path,
 * and hand the loaded graph to g2oc_upload as a g2oc_graph:
 *
 *   tag                            g2o type            line after the tag
 *   VERTEX_SE2                     VertexSE2           id x y theta
 *   EDGE_SE2                       EdgeSE2             id0 id1 x y theta  I (6, upper)
 *   VERTEX_SE3:QUAT                VertexSE3           id x y z qx qy qz qw
 *   EDGE_SE3:QUAT                  EdgeSE3             id0 id1 x y z qx qy qz qw  I (21, upper)
 *   VERTEX_SE3:EXPMAP              VertexSE3Expmap     id  (inverse of the estimate) tx ty tz qx qy qz qw
 *   VERTEX_TRACKXYZ                VertexPointXYZ      id x y z
 *   EDGE_PROJECT_XYZ2UV:EXPMAP     EdgeProjectXYZ2UV   id_point id_camera param_id u v  I (3, upper)
 *   EDGE_SE3:EXPMAP                EdgeSE3Expmap       id0 id1 (inverse of the measurement) tx ty tz qx qy qz qw
 *                                                      I (21, upper)
 *   PARAMS_CAMERAPARAMETERS        CameraParameters    id f cx cy baseline
 *   FIX                                                id id ...
 *
 * Entry points and the g2o functions they follow (paths relative to the g2o
 * source tree):
 *
 *   g2oc_file_load / g2oc_file_parse   OptimizableGraph::load(const char*) and
 *                                      load(istream) (g2o/core/optimizable_graph.cpp:344-531),
 *                                      with the types' read() (g2o/types/slam2d/vertex_se2.cpp:40-45,
 *                                      edge_se2.cpp:38-45, slam3d/vertex_se3.cpp:46-51,
 *                                      edge_se3.cpp:43-53, slam3d/vertex_pointxyz.cpp:40-42,
 *                                      sba/vertex_se3_expmap.cpp:35-40, sba/edge_project_xyz2uv.cpp:38-42,
 *                                      sba/edge_se3_expmap.cpp:33-43,
 *                                      sba/parameter_cameraparameters.cpp:43-49) and the
 *                                      "-renameTypes" lookup (optimizable_graph.cpp:619-644)
 *   g2oc_file_from_graph               a graph built in code (OptimizableGraph::addVertex /
 *                                      addEdge, g2o/core/optimizable_graph.cpp:179-246), to save
 *   g2oc_file_graph                    SparseOptimizer::initializeOptimization's vertex
 *                                      order (sorted by id) and edge order (insertion order)
 *   g2oc_file_fix_gauge                SparseOptimizer::gaugeFreedom + findGauge
 *                                      (g2o/core/sparse_optimizer.cpp:132-173) as g2o_cli
 *                                      applies them (g2o/apps/g2o_cli/g2o.cpp:303-339)
 *   g2oc_file_set_fixed                OptimizableGraph::Vertex::setFixed ("-gaugeList")
 *   g2oc_file_set_robust_huber         the "-robustKernel Huber -robustKernelWidth w
 *                                      [-nonSequential]" loop of g2o_cli (g2o.cpp:359-386)
 *   g2oc_file_set_estimates            the optimizer's result written back to the vertices
 *   g2oc_file_save                     OptimizableGraph::save / saveSubset(VertexSet) /
 *                                      saveSubset(EdgeSet) (optimizable_graph.cpp:533-610)
 *                                      with the types' write()
 *
 * Where this differs from g2o (all on malformed input):
 *   - A line whose numbers are missing or not finite numbers is refused and
 *     counted in lines_rejected (g2o adds the element with the values it got).
 *   - An edge whose vertices are of the wrong type for its tag is refused (g2o
 *     casts them unchecked).
 *   - Vertices are written in id order and edges in load order also by the two
 *     saveSubset forms (g2o writes those in pointer order).
 *   - The gauge is the vertex of maximum dimension with the lowest id (g2o takes
 *     the first such vertex of its hash map).
 */
#ifndef G2O_B200_G2O_IO_H
#define G2O_B200_G2O_IO_H

#include <stddef.h>
#include <stdint.h>

#include "g2o_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct g2oc_file g2oc_file;

typedef struct g2oc_file_info {
  int32_t num_vertices;       /* vertices loaded (poses and points) */
  int32_t num_edges;          /* edges loaded */
  int32_t num_parameters;     /* PARAMS_CAMERAPARAMETERS loaded */
  int32_t num_fixed;          /* vertices fixed now */
  int32_t lines;              /* lines read */
  int32_t lines_rejected;     /* element lines refused (see the header comment; g2o's "Failure
                                 adding Vertex", "Unable to find vertices", "Unable to add edge",
                                 "already defined" cases included) */
  int32_t lines_unsupported;  /* VERTEX_* / EDGE_* lines of tags the device path has no type for */
  int32_t lines_skipped;      /* other tags skipped (parameters, data, unknown types) */
  int32_t fix_not_found;      /* FIX ids with no vertex of that id loaded before the line */
  int32_t first_problem_line; /* line number of the first refused or unsupported line, 0: none */
  char first_problem[200];    /* its message */
} g2oc_file_info;

/* save modes */
#define G2OC_SAVE_ALL 0          /* OptimizableGraph::save: vertices of some edge, every edge */
#define G2OC_SAVE_VERTEX_SUBSET 1 /* saveSubset(VertexSet): the listed vertex ids, edges among them */
#define G2OC_SAVE_EDGE_SUBSET 2  /* saveSubset(EdgeSet): the listed edge indices (load order) and
                                    their vertices */

/* Load a .g2o file. renamed_types ("TAG_IN_FILE=TAG,TAG2=TAG3", or NULL) maps
   tags before they are looked up. Returns G2OC_OK with *out set (also for a
   file whose lines were all skipped: see g2oc_file_get_info), or
   G2OC_ERR_INVALID_ARGUMENT when the file cannot be opened. */
int g2oc_file_load(const char* path, const char* renamed_types, g2oc_file** out);
/* The same on text in memory (size bytes, no terminator needed). */
int g2oc_file_parse(const char* text, size_t size, const char* renamed_types, g2oc_file** out);
/* A file object holding a graph built in code (the vertices and edges a
   caller adds to an OptimizableGraph before save): pose_ids / point_ids give
   the vertex ids (NULL: poses 0..P-1, then points P..P+N-1); projection edges
   refer to one CameraParameters with id camera_param_id (baseline 0.5, the
   CameraParameters default). Robust deltas are kept. */
int g2oc_file_from_graph(const g2oc_graph* g, const int32_t* pose_ids, const int32_t* point_ids,
                         int32_t camera_param_id, g2oc_file** out);
void g2oc_file_free(g2oc_file* f);
int g2oc_file_get_info(const g2oc_file* f, g2oc_file_info* info);

/* The loaded graph as the C-ABI's structure of arrays: the vertices of the
   edges' types (poses, and points for projection edges), each sorted by id,
   edges in load order, Huber deltas if set. Vertices of other types have no
   edge and so are not in g2o's active set either; they are left out. The
   pointers stay valid until the next call on f that changes it, or
   g2oc_file_free. G2OC_ERR_BAD_GRAPH: no edge. G2OC_ERR_NOT_SUPPORTED: more
   than one edge type, or projection edges whose CameraParameters differ. */
int g2oc_file_graph(g2oc_file* f, g2oc_graph* out);
/* The vertex ids in g2oc_file_graph's order (num_poses / num_points each;
   either pointer may be NULL). */
int g2oc_file_vertex_ids(g2oc_file* f, int32_t* pose_ids, int32_t* point_ids);
/* Fix (fixed != 0) or free the vertex of that id. G2OC_ERR_INVALID_ARGUMENT: no such vertex. */
int g2oc_file_set_fixed(g2oc_file* f, int32_t id, int32_t fixed);
/* g2o_cli's gauge handling: if no vertex of the maximum dimension is fixed,
   fix the one with the lowest id and return its id in *gauge_id; otherwise
   *gauge_id = -1 ("fixed by priors or already fixed vertex"). */
int g2oc_file_fix_gauge(g2oc_file* f, int32_t* gauge_id);
/* Huber with this delta on every edge, or with non_sequential != 0 only on
   edges whose two vertex ids differ by more than one; delta <= 0 removes
   every robust kernel. */
int g2oc_file_set_robust_huber(g2oc_file* f, double delta, int32_t non_sequential);
/* Write estimates back in g2oc_file_graph's layout and order (as g2oc_download
   returns them); point_estimate may be NULL when there are no points. */
int g2oc_file_set_estimates(g2oc_file* f, const double* pose_estimate, const double* point_estimate);
/* Write the graph as g2o does (numbers with six significant digits). mode is a
   G2OC_SAVE_*; ids lists vertex ids or edge indices for the subset modes. */
int g2oc_file_save(const g2oc_file* f, const char* path, int32_t mode, const int32_t* ids, int32_t num_ids);

#ifdef __cplusplus
}
#endif

#endif /* G2O_B200_G2O_IO_H */
