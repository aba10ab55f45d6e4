/*
 * ref_driver.cu — TEST INFRASTRUCTURE ONLY.
 *
 * Driver for the reference FooskaGPU double-precision CUDA solver, compiled together with the
 * reference's own sources (mulitphase Solver/doublePrecision/*.cu except main.cu,
 * buildInput.cu, initialize.cu, explicitLoop.cu, export_plt.cu, restart.cu) by
 * oracle/build_ref.py into oracle/_ref/fooska_ref_dp.  It replaces only what the reference
 * hard-codes:
 *   - buildInput (DP/buildInput.cu:10): parameters come from a key = value case file with the
 *     INPUT field names;
 *   - initialize (DP/initialize.cu:61): the initial consVec comes from a binary file
 *     (nElem*10 doubles, .neu element order = local order with one rank);
 *   - explicitLoop (DP/explicitLoop.cu:3): the same call sequence, with a step cap, optional
 *     dumps of the stage-0 intermediates and CUDA-event timing of the step loop;
 *   - export_plt / readField / writeFieldRestart: not called (output is out of scope).
 * The mesh is read by the reference's translator from "sh.neu" in the working directory.
 *
 * usage: fooska_ref_dp <workdir> <case.txt> <ic.bin> <nsteps> [warmup] [--dump]
 * writes <workdir>/ref_U.bin (final consVec), ref_time.txt, and with --dump the stage-0
 * arrays ref_mesh_*.bin, ref_primF0.bin (before limiting), ref_primF.bin, ref_grad.bin,
 * ref_theta.bin, ref_wmin.bin, ref_wmax.bin, ref_rhs.bin, ref_dt.txt.
 */
#include <string>
#include <vector>

#include "strdata.h"

INPUT *d_input;
INPUT input;
int iStep = 0;
int iStart = 0;
double physicalTime = 0.0;
int printHLLC = 0;

static std::string g_icPath;

static void set_field(const std::string &k, double v) {
#define F(name) if (k == #name) { input.name = (decltype(input.name))v; return; }
    F(dt) F(cfl) F(adaptDt) F(adaptDtItr) F(maxDt) F(avfMin) F(rkSteps) F(finalTime) F(exportTime)
    F(restartStep) F(restartFlag) F(neglectX) F(neglectY) F(neglectZ) F(nMaterials) F(NEQ) F(scale)
    F(viscFlag) F(turbulence) F(woodsFlag) F(thermFntRlxFlag) F(thermRlxRate) F(thermUrf) F(thermItrMax)
    F(chemFlag) F(chemFntRlxFlag) F(chemRlxRate) F(chemUrf) F(chemItrMax) F(chemCondesation) F(chemLimit)
    F(consCalcFlag) F(consCalcIvar) F(satTempUrf)
#undef F
#define A(name) \
    if (k == #name "[0]") { input.name[0] = v; return; } \
    if (k == #name "[1]") { input.name[1] = v; return; }
    A(pInf) A(gamma) A(Cp) A(eta) A(satConst) A(dynVisc) A(heatCoef) A(Pr)
#undef A
    fprintf(stderr, "ref_driver: unknown case key %s\n", k.c_str());
    exit(3);
}

static void read_case(const char *path) {
    memset(&input, 0, sizeof(input));
    FILE *fp = fopen(path, "r");
    if (!fp) { fprintf(stderr, "ref_driver: cannot open %s\n", path); exit(2); }
    char line[512];
    while (fgets(line, sizeof line, fp)) {
        char key[128];
        double v;
        if (line[0] == '#') continue;
        if (sscanf(line, " %127[^= ] = %lf", key, &v) == 2) set_field(key, v);
    }
    fclose(fp);
}

/* replaces buildInput (DP/buildInput.cu:10-69) */
void buildInput() {
    cudaMalloc((void **)&d_input, sizeof(INPUT));
    cudaMemcpy(d_input, &input, sizeof(INPUT), cudaMemcpyHostToDevice);
}

/* replaces initialize (DP/initialize.cu:61-75) */
void initialize(int nElem, double *cellCenter, double *consVec) {
    (void)cellCenter;
    std::vector<double> h((size_t)nElem * 10);
    FILE *fp = fopen(g_icPath.c_str(), "rb");
    if (!fp || fread(h.data(), sizeof(double), h.size(), fp) != h.size()) {
        fprintf(stderr, "ref_driver: cannot read %zu doubles from %s\n", h.size(), g_icPath.c_str());
        exit(2);
    }
    fclose(fp);
    cudaMemcpy(consVec, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
}

void export_plt(EXPORT *exp, FIELD *field) { (void)exp; (void)field; }
void readField(int nElem, int rank, double *d_consVec) { (void)nElem; (void)rank; (void)d_consVec; }
void writeFieldRestart(int rank, MESH *mesh, FIELD *field) { (void)rank; (void)mesh; (void)field; }

template <typename X>
static void dump(const char *name, const X *dev, size_t n) {
    std::vector<X> h(n);
    cudaDeviceSynchronize();
    cudaMemcpy(h.data(), dev, n * sizeof(X), cudaMemcpyDeviceToHost);
    FILE *fp = fopen(name, "wb");
    fwrite(h.data(), sizeof(X), n, fp);
    fclose(fp);
}

int main(int argc, char **argv) {
    if (argc < 5) {
        fprintf(stderr, "usage: %s <workdir> <case.txt> <ic.bin> <nsteps> [warmup] [--dump]\n", argv[0]);
        return 1;
    }
    std::string caseAbs = argv[2], icAbs = argv[3];
    if (chdir(argv[1]) != 0) { fprintf(stderr, "ref_driver: bad workdir\n"); return 2; }
    read_case(caseAbs.c_str());
    g_icPath = icAbs;
    const int nSteps = atoi(argv[4]);
    const int warm = (argc > 5 && argv[5][0] != '-') ? atoi(argv[5]) : 0;
    bool doDump = false;
    for (int i = 5; i < argc; i++) if (std::string(argv[i]) == "--dump") doDump = true;

    MPI_Init(&argc, &argv);
    cudaSetDevice(0);
    MESH *mesh = (MESH *)malloc(sizeof(MESH));
    FIELD *field = (FIELD *)malloc(sizeof(FIELD));
    EXPORT *exp = (EXPORT *)malloc(sizeof(EXPORT));
    COMM *comm = (COMM *)malloc(sizeof(COMM));
    buildInput();
    mainStart(mesh, exp, comm, field);

    const int nE = mesh->nElem, nF = mesh->nFcs;
    if (doDump) {
        dump("ref_mesh_fc2el.bin", mesh->fc2el, (size_t)nF * 2);
        dump("ref_mesh_bc.bin", mesh->boundCond, (size_t)nF);
        dump("ref_mesh_n.bin", mesh->n, (size_t)nF * 3);
        dump("ref_mesh_nt1.bin", mesh->nt1, (size_t)nF * 3);
        dump("ref_mesh_nt2.bin", mesh->nt2, (size_t)nF * 3);
        dump("ref_mesh_area.bin", mesh->area, (size_t)nF);
        dump("ref_mesh_vol.bin", mesh->volume, (size_t)nE);
        dump("ref_mesh_cc.bin", mesh->cellCenter, (size_t)nE * 3);
        dump("ref_mesh_fc.bin", mesh->fcCenter, (size_t)nF * 3);
    }

    /* explicitLoop (DP/explicitLoop.cu:3-64) with a step cap */
    cudaDeviceSynchronize();
    cudaEvent_t evInitGrads, evGreenGauss, evCompLimiter, evInitRHS, evFluxDone, evStepDone, t0, t1;
    cudaEventCreate(&evInitGrads);
    cudaEventCreate(&evGreenGauss);
    cudaEventCreate(&evCompLimiter);
    cudaEventCreate(&evInitRHS);
    cudaEventCreate(&evFluxDone);
    cudaEventCreate(&evStepDone);
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaStream_t sMain, sProx;
    cudaStreamCreateWithFlags(&sMain, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&sProx, cudaStreamNonBlocking);
    iStep = 0;
    for (int s = 0; s < nSteps + warm; s++) {
        if (s == warm) { cudaDeviceSynchronize(); cudaEventRecord(t0, 0); }
        physicalTime += input.dt;
        if (input.rkSteps > 1) initRk(mesh, field, sMain);
        for (int irk = 0; irk < input.rkSteps; irk++) {
            recvArray(comm, 0, 10, comm->recvbuff);
            recvArray(comm, 1, 10, comm->recvbuff);
            recvArray(comm, 2, 3 * 3, comm->recvBuffGrad);
            computePrimVec(mesh, field, comm, sMain, sProx);
            if (doDump && s == 0 && irk == 0) dump("ref_primF0.bin", field->primVecF, (size_t)nF * 20);
            computeGrad(mesh, field, comm, sMain, sProx, evInitGrads, evGreenGauss);
            computeFaceValues(mesh, field, comm, sMain, sProx, evGreenGauss, evCompLimiter);
            computeRHS(mesh, field, comm, sMain, sProx, evInitRHS, evFluxDone);
            if (doDump && s == 0 && irk == 0) {
                dump("ref_primF.bin", field->primVecF, (size_t)nF * 20);
                dump("ref_grad.bin", field->grad, (size_t)nE * 30);
                dump("ref_theta.bin", field->theta, (size_t)nE * 10);
                dump("ref_wmin.bin", field->wMin, (size_t)nE * 10);
                dump("ref_wmax.bin", field->wMax, (size_t)nE * 10);
                dump("ref_rhs.bin", field->RHS, (size_t)nE * 10);
            }
            if (input.adaptDt == 1 && irk == 0 && iStep % input.adaptDtItr == 0) {
                computeTimeStep(mesh, field, comm, sMain, sProx);
                if (doDump && s == 0) {
                    FILE *fp = fopen("ref_dt.txt", "w");
                    fprintf(fp, "%.17g\n", input.dt);
                    fclose(fp);
                }
            }
            update(irk, mesh, field, sMain, sProx, evFluxDone, evStepDone);
        }
        relaxation(mesh, field, comm, sMain, sProx, evStepDone);
        if (input.consCalcFlag == 1 && iStep % input.adaptDtItr == 0) consCalc(mesh, field, sMain);
        iStep++;
    }
    // the stage functions run on the non-blocking streams sMain / sProx: wait for all of them
    // before the end event, so the last stage's update and relaxation are inside the timed region
    cudaDeviceSynchronize();
    cudaEventRecord(t1, 0);
    cudaEventSynchronize(t1);
    float ms = 0;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaError_t err = cudaGetLastError();
    dump("ref_U.bin", field->consVec, (size_t)nE * 10);
    FILE *fp = fopen("ref_time.txt", "w");
    fprintf(fp, "%d %d %.6f %.17g %.17g %s\n", nE, nSteps, ms, physicalTime, input.dt,
            err == cudaSuccess ? "ok" : cudaGetErrorString(err));
    fclose(fp);
    printf("ref_driver: %d cells, %d steps, %.3f ms, %s\n", nE, nSteps, ms, cudaGetErrorString(err));
    MPI_Finalize();
    return err == cudaSuccess ? 0 : 4;
}
