// chfem_exec.cpp -- command-line front end of chfem_b200, with the flags of chfem's
// chfem_exec (chfem/src/main.c:155-323): [.nf] [.raw] -b -c -d -e -f -h -i -j -m -p -pm -r
// -s -u -xi -xo, plus --precision {fp64,mixed} and --multirhs (no counterpart in the
// reference).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/chfem_b200.h"

static void help() {
  printf("\nchfem_b200 -- computational homogenization with the image-based FEM on B200\n\n");
  printf("./chfem_exec [.nf] [.raw] ... (options)\n\nor\n\n./chfem_exec (options) ... -i [.nf] [.raw] ... (options)\n\n");
  printf("\t-b: Save results in a binary file. Must be followed by a string with a filename.\n");
  printf("\t-c: Stopping criteria for the PCG method: 0 - L2 (default), 1 - Inf, 2 - L2+Error.\n");
  printf("\t-d: Target direction: 0 - X, 1 - Y, 2 - Z, 3 - YZ, 4 - XZ, 5 - XY, 6 - ALL (default).\n");
  printf("\t-e: Export fields from simulation (by nodes).\n");
  printf("\t-f: Input scalar density field (not provided by chfem_b200).\n");
  printf("\t-h: Print this help info and exit.\n");
  printf("\t-i: Input files. Must be followed by: [.nf] [.raw].\n");
  printf("\t-j: Jacobi preconditioning: 0 - no, 1 - yes (default).\n");
  printf("\t-m: Write metrics report. Must be followed by a string with a filename.\n");
  printf("\t-p: Parallel matrix-free strategy: 0 - NBN (default), 1 - EBE.\n");
  printf("\t-pm: Pore mapping strategy: 0 - image, 1 - DOF number (default).\n");
  printf("\t-r: Number of recursive searches for initial guesses.\n");
  printf("\t-s: Solver: 0 - CG (default), 1 - MINRES, 2 - CG3, 3 - MINRES3, 4 - CG2, 5 - MINRES2.\n");
  printf("\t-u: Reduce strategy for velocity fields (FLUID): 0 - on the fly, 1 - only diag, 2 - full.\n");
  printf("\t-xi: Import initial guesses for PCG solver from binary files. Must be followed by a string with a filename.\n");
  printf("\t-xo: Export result vector (x) from the PCG solver.\n");
  printf("\t--precision fp64|mixed: arithmetic of the solver (default fp64).\n\n");
}

int main(int argc, char** argv) {
  if (argc < 2) { printf("Invalid input.\nCall -h for help with input directives.\n"); return 0; }
  for (int i = 1; i < argc; i++)
    if (!strcmp(argv[i], "-h")) { help(); return 0; }
  const char *nf = nullptr, *raw = nullptr, *bin = nullptr, *report = nullptr, *x0 = nullptr, *sdf = nullptr;
  unsigned dir = 6, solver = 0, precond = 1, par = 0, poremap = 1, recursions = 0, stopcrit = 0, xreduce = 2;
  int export_fields = 0, export_x = 0, precision = 0, multirhs = 0;
  int id = 0;
  for (int i = 1; i < argc; i++) if (!strcmp(argv[i], "-i")) { id = i; break; }
  if (id) { if (id + 2 >= argc) { printf("Invalid input after -i.\n"); return 0; } nf = argv[id + 1]; raw = argv[id + 2]; }
  else { if (argc < 3) { printf("Invalid input ignored: %s.\nCall -h for help with input directives.\n", argv[1]); return 0; } nf = argv[1]; raw = argv[2]; }
  for (int i = id ? 1 : 3; i < argc; i++) {
    if (id && i == id) { i += 2; continue; }
    auto next = [&](const char* f) -> const char* {
      if (i + 1 >= argc) { printf("Invalid input after %s.\nCall -h for help with input directives.\n", f); exit(0); }
      return argv[++i];
    };
    const char* a = argv[i];
    if (!strcmp(a, "-r")) recursions = atoi(next(a));
    else if (!strcmp(a, "-j")) precond = atoi(next(a));
    else if (!strcmp(a, "-u")) xreduce = atoi(next(a));
    else if (!strcmp(a, "-s")) solver = atoi(next(a));
    else if (!strcmp(a, "-p")) par = atoi(next(a));
    else if (!strcmp(a, "-pm")) poremap = atoi(next(a));
    else if (!strcmp(a, "-d")) dir = atoi(next(a));
    else if (!strcmp(a, "-c")) stopcrit = atoi(next(a));
    else if (!strcmp(a, "-e")) export_fields = 1;
    else if (!strcmp(a, "-b")) bin = next(a);
    else if (!strcmp(a, "-f")) sdf = next(a);
    else if (!strcmp(a, "-m")) report = next(a);
    else if (!strcmp(a, "-xi")) x0 = next(a);
    else if (!strcmp(a, "-xo")) export_x = 1;
    else if (!strcmp(a, "--precision")) precision = !strcmp(next(a), "mixed");
    else if (!strcmp(a, "--multirhs")) multirhs = 1;
    else printf("Invalid input ignored: %s.\n", a);
  }
  int ok = 1;
  if (xreduce > 2) { printf("Invalid reduce strategy flag.\n"); ok = 0; }
  if (solver > 5) { printf("Invalid solver flag.\n"); ok = 0; }
  if (par > 1) { printf("Invalid parallel strategy flag.\n"); ok = 0; }
  if (!ok) { printf("Call -h for help with input directives.\n"); return 0; }

  printf("#######################################################\n");
  chfemB200SetPrecision(precision);
  chfemB200SetMultiRHS(multirhs);
  if (!hmgInit((char*)nf, (char*)raw, (char*)sdf, nullptr)) {
    printf("Failed to properly read input files.\nProcess aborted.\n#######################################################\n");
    return -1;
  }
  // main.c:72-152
  if (report) hmgKeepTrackOfAnalysisReport(1);
  hmgSaveFields((logical)export_fields, 0);
  hmgSetParallelStrategyFlag((uint8_t)par);
  if (!hmgSetPoreMappingStrategy((uint8_t)poremap)) { printf("ERROR: Failed to set \"poremap_flag\"=%u.\nProcess aborted.\n", poremap); hmgEnd(); return -1; }
  hmgSetSolverFlag((uint8_t)solver);
  hmgSetPreConditionerFlag((uint8_t)precond);
  hmgSetXReduceFlag((uint8_t)xreduce);
  hmgSetHomogenizationFlag((hmgFlag_t)dir);
  hmgPrintModelData();
  hmgSetStoppingCriteria((uint8_t)stopcrit);
  if (x0) hmgImportX((char*)x0);
  else hmgFindInitialGuesses(recursions);
  hmgExportX((logical)export_x);
  hmgSolveHomogenization();
  if (chfemB200LastError()[0]) { printf("Failed to run analysis: %s\nProcess aborted.\n", chfemB200LastError()); hmgEnd(); return -1; }
  hmgPrintConstitutiveMtx();
  hmgPrintReport(report);
  if (bin) hmgSaveConstitutiveMtx(bin);
  hmgEnd();
  printf("#######################################################\n");
  return 0;
}
