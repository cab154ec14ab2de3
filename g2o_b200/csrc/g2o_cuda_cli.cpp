// g2o_cuda_cli.cpp -- command-line optimizer for .g2o files on the device
// path: g2o_cli (g2o/apps/g2o_cli/g2o.cpp:100-740) restricted to what the
// backend optimizes, through the C-ABI only (include/g2o_cuda.h,
// include/g2o_io.h).
//
//   g2o_cuda_cli [-i N] [-v] [-solver lm_cuda] [-o out.g2o] [-stats f] [-summary f]
//                [-robustKernel Huber] [-robustKernelWidth w] [-nonSequential]
//                [-gaugeList 1,2] [-renameTypes A=B,...] [-solverProperties k=v,...]
//                [-gain g] [-ig n] [-device d] [-computeMarginals] [-listSolvers]
//                [-listRobustKernels] [-printSolverProperties] graph.g2o | -
//
// Messages go to stderr with g2o_cli's wording; exit codes follow it (1: no
// vertices or the file cannot be opened, 2: load error, 3: the solver does
// not suit the graph). Options of g2o_cli outside the device path (-guess,
// -guessOdometry, -inc, -update, -guiout, -gnudump) are refused with exit
// code 1. -computeMarginals prints the blocks (h, h) and (h-1, h) of Hpp^-1
// for every free pose h, as g2o_cli does (g2o.cpp:620-652).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <iterator>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/g2o_cuda.h"
#include "../../include/g2o_io.h"

namespace {

struct Args {
  int iterations = 5;
  bool verbose = false;
  std::string solver = "gn_cuda";
  std::string output, stats, summary, robust, gauge_list, renames, properties, input;
  double robust_width = -1.0;
  bool non_sequential = false;
  double gain = 1e-6;
  int max_iterations_with_gain = std::numeric_limits<int>::max();
  int device = 0;
  bool list_solvers = false, list_kernels = false, list_types = false, print_properties = false;
  bool marginalize = false;  // accepted: the points of a projection graph are always marginalized
  bool marginals = false;
};

const char* const kRefused[] = {"-guess", "-guessOdometry", "-inc", "-update", "-guiout", "-gnudump",
                                "-gaugeId"};

int usage(const char* msg) {
  std::cerr << msg << "\nusage: g2o_cuda_cli [options] graph.g2o (see the source header for the options)\n";
  return 1;
}

// g2o's CommandArgs: "-name value", bool flags without a value, one left-over
// argument (the graph file)
bool parse_args(int argc, char** argv, Args& a, std::string& err) {
  for (int i = 1; i < argc; ++i) {
    const std::string s = argv[i];
    auto value = [&](std::string& out) {
      if (i + 1 >= argc) {
        err = "missing value for " + s;
        return false;
      }
      out = argv[++i];
      return true;
    };
    std::string v;
    for (const char* r : kRefused)
      if (s == r) {
        err = s + " is not supported by the device path";
        return false;
      }
    if (s == "-i") {
      if (!value(v)) return false;
      a.iterations = std::atoi(v.c_str());
    } else if (s == "-v") a.verbose = true;
    else if (s == "-solver") { if (!value(a.solver)) return false; }
    else if (s == "-o") { if (!value(a.output)) return false; }
    else if (s == "-stats") { if (!value(a.stats)) return false; }
    else if (s == "-summary") { if (!value(a.summary)) return false; }
    else if (s == "-robustKernel") { if (!value(a.robust)) return false; }
    else if (s == "-robustKernelWidth") {
      if (!value(v)) return false;
      a.robust_width = std::atof(v.c_str());
    } else if (s == "-nonSequential") a.non_sequential = true;
    else if (s == "-gaugeList") { if (!value(a.gauge_list)) return false; }
    else if (s == "-renameTypes") { if (!value(a.renames)) return false; }
    else if (s == "-solverProperties") { if (!value(a.properties)) return false; }
    else if (s == "-gain") {
      if (!value(v)) return false;
      a.gain = std::atof(v.c_str());
    } else if (s == "-ig") {
      if (!value(v)) return false;
      a.max_iterations_with_gain = std::atoi(v.c_str());
    } else if (s == "-device") {
      if (!value(v)) return false;
      a.device = std::atoi(v.c_str());
    } else if (s == "-solverlib" || s == "-typeslib") {
      if (!value(v)) return false;  // the device solvers and types are built in
    } else if (s == "-listSolvers") a.list_solvers = true;
    else if (s == "-listRobustKernels") a.list_kernels = true;
    else if (s == "-listTypes") a.list_types = true;
    else if (s == "-printSolverProperties") a.print_properties = true;
    else if (s == "-marginalize") a.marginalize = true;
    else if (s == "-computeMarginals") a.marginals = true;
    else if (s.size() > 1 && s[0] == '-') {
      err = "unknown option " + s;
      return false;
    } else {
      a.input = s;
    }
  }
  return true;
}

std::vector<std::string> split(const std::string& s, char d) {
  std::vector<std::string> out;
  std::string cur;
  std::istringstream is(s);
  while (std::getline(is, cur, d)) out.push_back(cur);
  return out;
}

std::string trim(const std::string& s) {
  const size_t b = s.find_first_not_of(" \t\n");
  if (b == std::string::npos) return "";
  return s.substr(b, s.find_last_not_of(" \t\n") - b + 1);
}

// "-solverProperties name=value,..." with the property names of
// OptimizationAlgorithmLevenberg (optimization_algorithm_levenberg.cpp:42-58)
// and LinearSolverPCG (linear_solver_pcg.h:45-50)
bool apply_properties(const std::string& spec, g2oc_params& p) {
  bool ok = true;
  for (const std::string& item : split(spec, ',')) {
    const std::vector<std::string> kv = split(item, '=');
    if (kv.size() != 2) continue;
    const std::string k = trim(kv[0]), v = trim(kv[1]);
    if (k == "initialLambda") p.initial_lambda = std::atof(v.c_str());
    else if (k == "tau") p.tau = std::atof(v.c_str());
    else if (k == "maxTrialsAfterFailure") p.max_trials_after_failure = std::atoi(v.c_str());
    else if (k == "initialDelta") p.initial_delta = std::atof(v.c_str());
    else if (k == "lambdaFactor") p.lambda_factor = std::atof(v.c_str());
    else if (k == "tolerance") p.pcg_tolerance = std::atof(v.c_str());
    else if (k == "maxIterations") p.pcg_max_iterations = std::atoi(v.c_str());
    else if (k == "absoluteTolerance") p.pcg_absolute_tolerance = (v == "1" || v == "true");
    else {
      std::cerr << "unknown solver property " << k << std::endl;
      ok = false;
    }
  }
  return ok;
}

void print_properties(const g2oc_params& p) {
  std::cerr << "initialLambda " << p.initial_lambda << "\ntau " << p.tau << "\nmaxTrialsAfterFailure "
            << p.max_trials_after_failure << "\ntolerance " << p.pcg_tolerance << "\nmaxIterations "
            << p.pcg_max_iterations << "\nabsoluteTolerance " << p.pcg_absolute_tolerance << std::endl;
}

// G2OBatchStatistics' operator<< (g2o/core/batch_stats.cpp:48-84), one line per iteration
void write_stats_line(std::ostream& os, const g2oc_iteration_stats& s, int nv, int ne, const g2oc_hessian_info& h) {
#define PTH(name, val) os << name << "= " << (val) << "\t "
  PTH("iteration", s.iteration);
  PTH("numVertices", nv);
  PTH("numEdges", ne);
  PTH("chi2", s.chi2);
  PTH("timeResiduals", s.time_residuals);
  PTH("timeLinearize", 0);
  PTH("timeQuadraticForm", s.time_quadratic_form);
  PTH("timeSchurComplement", s.time_schur_complement);
  PTH("timeSymbolicDecomposition", 0);
  PTH("timeNumericDecomposition", 0);
  PTH("timeLinearSolution", s.time_linear_solver);
  PTH("iterationsLinearSolver", s.iterations_linear_solver);
  PTH("timeUpdate", s.time_update);
  PTH("timeIteration", s.time_iteration);
  PTH("levenbergIterations", s.levenberg_iterations);
  PTH("timeLinearSolver", s.time_linear_solver);
  PTH("hessianDimension", h.vector_size);
  PTH("hessianPoseDimension", (int64_t)h.num_free_poses * h.pose_dim);
  PTH("hessianLandmarkDimension", (int64_t)h.num_free_points * h.point_dim);
  PTH("choleskyNNZ", 0);
  PTH("timeMarginals", 0);
#undef PTH
}

std::string fixed6(double v) {
  char b[64];
  std::snprintf(b, sizeof(b), "%f", v);
  return b;
}

}  // namespace

int main(int argc, char** argv) {
  Args a;
  std::string err;
  if (!parse_args(argc, argv, a, err)) return usage(err.c_str());
  if (a.list_solvers) {
    std::vector<char> buf(4096);
    g2oc_list_solvers(buf.data(), buf.size());
    for (const std::string& n : split(buf.data(), ';'))
      if (!n.empty()) std::cout << n << std::endl;
    return 0;
  }
  if (a.list_types) {
    std::cout << "VERTEX_SE2\nEDGE_SE2\nVERTEX_SE3:QUAT\nEDGE_SE3:QUAT\nVERTEX_SE3:EXPMAP\nVERTEX_TRACKXYZ\n"
                 "EDGE_PROJECT_XYZ2UV:EXPMAP\nPARAMS_CAMERAPARAMETERS\n";
    return 0;
  }
  if (a.list_kernels) {
    std::cout << "Huber" << std::endl;
    return 0;
  }
  g2oc_params params;
  if (g2oc_construct(a.solver.c_str(), &params) != G2OC_OK) {
    std::cerr << "Error allocating solver. Allocating \"" << a.solver << "\" failed!" << std::endl;
    return 0;
  }
  if (!a.properties.empty() && !apply_properties(a.properties, params)) return 1;
  if (a.print_properties || !a.properties.empty()) print_properties(params);

  bool gain_mode = false;
  if (a.iterations < 0) {
    std::cerr << "# setup termination criterion based on the gain of the iteration" << std::endl;
    a.iterations = a.max_iterations_with_gain;
    gain_mode = true;
  }

  // loading (g2o.cpp:263-292)
  if (a.input.empty()) {
    std::cerr << "No input data specified" << std::endl;
    return 0;
  }
  g2oc_file* file = nullptr;
  const char* ren = a.renames.empty() ? nullptr : a.renames.c_str();
  if (a.input == "-") {
    std::cerr << "Read input from stdin" << std::endl;
    std::string text((std::istreambuf_iterator<char>(std::cin)), std::istreambuf_iterator<char>());
    if (g2oc_file_parse(text.data(), text.size(), ren, &file) != G2OC_OK) {
      std::cerr << "Error loading graph" << std::endl;
      return 2;
    }
  } else {
    std::cerr << "Read input from " << a.input << std::endl;
    if (g2oc_file_load(a.input.c_str(), ren, &file) != G2OC_OK) {
      std::cerr << "Failed to open file" << std::endl;
      return 1;
    }
  }
  g2oc_file_info info;
  g2oc_file_get_info(file, &info);
  if (info.first_problem_line)
    std::cerr << "# " << info.lines_rejected << " lines refused, " << info.lines_unsupported
              << " of unsupported types; first: " << info.first_problem << std::endl;
  std::cerr << "Loaded " << info.num_vertices << " vertices" << std::endl;
  std::cerr << "Loaded " << info.num_edges << " edges" << std::endl;
  if (info.num_vertices == 0) {
    std::cerr << "Graph contains no vertices" << std::endl;
    g2oc_file_free(file);
    return 1;
  }
  if (info.lines_unsupported > 0) {
    std::cerr << "The selected solver is not suitable for optimizing the given graph" << std::endl;
    g2oc_file_free(file);
    return 3;
  }

  // gauge (g2o.cpp:303-339)
  if (!a.gauge_list.empty()) {
    std::cerr << "Fixing gauges: ";
    for (const std::string& t : split(a.gauge_list, ',')) {
      const int id = std::atoi(t.c_str());
      if (g2oc_file_set_fixed(file, id, 1) != G2OC_OK) {
        std::cerr << "fatal, not found the vertex of id " << id << " in the gaugeList. Aborting";
        g2oc_file_free(file);
        return -1;
      }
      std::cerr << id << " ";
    }
    std::cerr << std::endl;
  } else {
    int32_t gid = -1;
    g2oc_file_fix_gauge(file, &gid);
    if (gid >= 0) std::cerr << "# graph is fixed by node " << gid << std::endl;
    else std::cerr << "# graph is fixed by priors or already fixed vertex" << std::endl;
  }

  // robust kernel (g2o.cpp:359-386)
  if (!a.robust.empty()) {
    if (a.robust != "Huber") {
      std::cerr << "Robust kernel " << a.robust << " is not supported by the device path (Huber only)" << std::endl;
      g2oc_file_free(file);
      return 1;
    }
    std::cerr << "# Preparing robust error function ... ";
    g2oc_file_set_robust_huber(file, a.robust_width > 0 ? a.robust_width : 1.0, a.non_sequential ? 1 : 0);
    std::cerr << "done." << std::endl;
  }

  g2oc_graph graph;
  int st = g2oc_file_graph(file, &graph);
  if (st != G2OC_OK) {
    std::cerr << g2oc_last_error() << std::endl;
    std::cerr << "The selected solver is not suitable for optimizing the given graph" << std::endl;
    g2oc_file_free(file);
    return 3;
  }
  if (graph.num_points > 0) std::cerr << "# Preparing Marginalization of the Landmarks ... done." << std::endl;
  const int nv = graph.num_poses + graph.num_points, ne = graph.num_edges;
  std::vector<g2oc_iteration_stats> stats;
  g2oc_hessian_info hinfo;
  std::memset(&hinfo, 0, sizeof(hinfo));
  double load_chi = 0.0, final_chi = 0.0;
  int result_iterations = 0;

  g2oc_ctx* ctx = nullptr;
  st = g2oc_create(a.device, &ctx);
  if (st != G2OC_OK) {
    if (a.iterations != 0) {
      std::cerr << "no usable CUDA device: " << g2oc_last_error() << std::endl;
      g2oc_file_free(file);
      return 1;
    }
    std::cerr << "# no CUDA device: the graph is not uploaded (0 iterations)" << std::endl;
  } else {
    if ((st = g2oc_set_params(ctx, &params)) != G2OC_OK || (st = g2oc_upload(ctx, &graph)) != G2OC_OK) {
      std::cerr << "upload failed: " << g2oc_last_error() << std::endl;
      g2oc_destroy(ctx);
      g2oc_file_free(file);
      return 3;
    }
    g2oc_get_hessian_info(ctx, &hinfo);
    double rchi;
    g2oc_chi2(ctx, &load_chi, &rchi);
    std::cerr << "Initial chi2 = " << fixed6(load_chi) << std::endl;
    // SparseOptimizer::optimize (sparse_optimizer.cpp:393-455) with the
    // gain-based SparseOptimizerTerminateAction when -i is negative
    // (g2o/core/sparse_optimizer_terminate_action.cpp:50-85)
    double cum = 0.0, last_chi = 0.0;
    int result = G2OC_RESULT_OK;
    bool fail = false;
    for (int i = 0; i < a.iterations && result == G2OC_RESULT_OK; ++i) {
      g2oc_iteration_stats s;
      std::memset(&s, 0, sizeof(s));
      st = g2oc_iterate(ctx, i, &s, &result);
      if (st != G2OC_OK) {
        std::cerr << "iteration " << i << " failed: " << g2oc_last_error() << std::endl;
        fail = true;
        break;
      }
      stats.push_back(s);
      ++result_iterations;
      if (a.verbose) {
        cum += s.time_iteration;
        std::cerr << "iteration= " << i << "\t chi2= " << fixed6(s.chi2) << "\t time= " << s.time_iteration
                  << "\t cumTime= " << cum << "\t edges= " << hinfo.num_active_edges;
        if (params.algorithm != G2OC_ALGO_DOGLEG) std::cerr << "\t schur= " << (hinfo.num_free_points > 0 ? 1 : 0);
        if (params.algorithm == G2OC_ALGO_LEVENBERG)
          std::cerr << "\t lambda= " << fixed6(s.lambda) << "\t levenbergIter= " << s.levenberg_iterations;
        if (params.algorithm == G2OC_ALGO_DOGLEG) {
          // OptimizationAlgorithmDogleg::printVerbose (optimization_algorithm_dogleg.cpp:182-187)
          static const char* const kStep[] = {"Undefined", "Descent", "GN", "Dogleg"};
          std::cerr << "\t Delta= " << s.trust_radius << "\t step= " << kStep[s.dogleg_step & 3]
                    << "\t tries= " << s.levenberg_iterations;
          if (s.lambda > 0) std::cerr << "\t lambda= " << s.lambda;
        }
        std::cerr << std::endl;
      }
      if (gain_mode) {
        if (i == 0) last_chi = s.chi2;
        else {
          const double gain = (last_chi - s.chi2) / s.chi2;
          last_chi = s.chi2;
          if (gain >= 0 && gain < a.gain) break;
        }
      }
    }
    if (result == G2OC_RESULT_FAIL || fail) {
      result_iterations = 0;
      if (a.iterations > 0) std::cerr << "Cholesky failed, result might be invalid" << std::endl;
    } else if (a.marginals) {
      // free poses in Hessian order: pose ids ascending, fixed ones skipped
      std::vector<int32_t> ids(graph.num_poses), hid;
      g2oc_file_vertex_ids(file, ids.data(), nullptr);
      for (int i = 0; i < graph.num_poses; ++i)
        if (!(graph.pose_fixed && graph.pose_fixed[i])) hid.push_back(ids[i]);
      std::vector<int32_t> req;
      for (int h = 0; h < (int)hid.size(); ++h) {
        req.push_back(h); req.push_back(h);
        if (h > 0) { req.push_back(h - 1); req.push_back(h); }
      }
      const int pd = hinfo.pose_dim, nreq = (int)req.size() / 2;
      std::vector<double> blocks((size_t)nreq * pd * pd);
      if (g2oc_compute_marginals(ctx, nreq, req.data(), blocks.data()) == G2OC_OK) {
        for (int q = 0; q < nreq; ++q) {
          const int r = req[2 * q], cc = req[2 * q + 1];
          if (r == cc) std::cerr << "Vertex id:" << hid[r] << std::endl;
          std::cerr << "inv block :" << r << ", " << cc << std::endl;
          for (int i = 0; i < pd; ++i) {
            for (int j = 0; j < pd; ++j) std::cerr << (j ? " " : "") << blocks[((size_t)q * pd + i) * pd + j];
            std::cerr << std::endl;
          }
        }
      } else {
        std::cerr << "computing the marginals failed: " << g2oc_last_error() << std::endl;
      }
    }
    std::vector<double> pose((size_t)graph.num_poses * (graph.pose_type == G2OC_POSE_SE2 ? 3
                                                        : graph.pose_type == G2OC_POSE_SE3 ? 12 : 7));
    std::vector<double> point((size_t)graph.num_points * 3);
    g2oc_download(ctx, pose.data(), point.empty() ? nullptr : point.data());
    g2oc_chi2(ctx, &final_chi, &rchi);
    g2oc_destroy(ctx);
    g2oc_file_set_estimates(file, pose.data(), point.empty() ? nullptr : point.data());
  }

  if (!a.summary.empty()) {
    // PropertyMap::writeToCSV of g2o_cli's summary (g2o.cpp:658-702), names in map order
    FILE* fp = std::fopen(a.summary.c_str(), "a");
    if (fp) {
      const char* etag = graph.edge_type == G2OC_EDGE_SE2 ? "EDGE_SE2"
                         : graph.edge_type == G2OC_EDGE_SE3 ? "EDGE_SE3:QUAT" : "EDGE_PROJECT_XYZ2UV:EXPMAP";
      std::fprintf(fp, "edge_types,filename,final_chi,init_chi,load_chi,maxIterations,n_edges,n_landmarks,n_poses,"
                       "n_vertices,realIterations,robustKernel,solver\n");
      std::fprintf(fp, "%s ,%s,%g,%g,%g,%d,%d,%d,%d,%d,%d,%d,%s\n", etag, a.input.c_str(), final_chi, load_chi,
                   load_chi, a.iterations, info.num_edges, graph.num_points, graph.num_poses, info.num_vertices,
                   result_iterations, a.robust.empty() ? 0 : 1, a.solver.c_str());
      std::fclose(fp);
    }
  }
  if (!a.stats.empty()) {
    std::cerr << "writing stats to file \"" << a.stats << "\" ... ";
    FILE* fp = std::fopen(a.stats.c_str(), "w");
    if (fp) {
      for (const g2oc_iteration_stats& s : stats) {
        std::ostringstream os;
        write_stats_line(os, s, nv, ne, hinfo);
        std::fprintf(fp, "%s\n", os.str().c_str());
      }
      std::fclose(fp);
    }
    std::cerr << "done." << std::endl;
  }
  if (!a.output.empty()) {
    if (a.output == "-") {
      std::cerr << "saving to stdout";
      g2oc_file_save(file, "/dev/stdout", G2OC_SAVE_ALL, nullptr, 0);
    } else {
      std::cerr << "saving " << a.output << " ... ";
      if (g2oc_file_save(file, a.output.c_str(), G2OC_SAVE_ALL, nullptr, 0) != G2OC_OK)
        std::cerr << g2oc_last_error() << " ";
    }
    std::cerr << "done." << std::endl;
  }
  g2oc_file_free(file);
  return 0;
}
