/*
 * C-ABI harness over the DynELA reference (test infrastructure only).
 *
 * This file is compiled together with the reference's own sources (see the
 * Makefile beside it) into oracle/_ref/libdnlref.so.  It builds a reference
 * model from the same `dnl_model_desc` the engine takes, runs the reference's
 * own per-increment methods, and exposes the reference state (nodes, nodal
 * fields, integration points) as plain arrays so that tests can compare the
 * CPU restatement and the GPU engine with the real thing, and so that the
 * reference CPU path can be timed as a baseline.
 *
 * Only one harness model may be alive at a time: the reference keeps its model
 * in the global `dynelaData` (Sources/dnlFEM/DynELA.C:21-47).
 */
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <string>
#include <vector>
#include <unistd.h>
#include <chrono>
#include <sstream>
#include <regex>
#include <complex>
#include <memory>
#include <numeric>
#include <iomanip>
#include <ostream>
#include <typeinfo>
#include <stdexcept>
#include <cassert>
#include <ctime>
#include <strings.h>
#include <string.h>
#include <stdint.h>
#include <libgen.h>
#include <pwd.h>
#include <omp.h>
#include <zlib.h>
#include <ifaddrs.h>

// The harness reads and writes reference state that the classes keep private
// (solver parameters, the end time of the current solve); the reference
// sources themselves are compiled unchanged.
#define private public
#define protected public
#include <DynELA.h>
#include <Explicit.h>
#include <Model.h>
#include <Element.h>
#include <Node.h>
#include <NodalField.h>
#include <NodeSet.h>
#include <ElementSet.h>
#include <Material.h>
#include <JohnsonCookLaw.h>
#include <IntegrationPoint.h>
#include <BoundaryRestrain.h>
#include <BoundarySpeed.h>
#include <DiscreteFunction.h>
#include <ElQua4NAx.h>
#include <ElQua4N2D.h>
#include <ElHex8N3D.h>
#include <Timer.h>
#undef private
#undef protected

#include "dnlgpu.h"

extern DynELA *dynelaData;

namespace
{
struct RefModel
{
  DynELA *dyn = nullptr;
  Explicit *solver = nullptr;
  int type = 0, npe = 0, dim = 0;
  long nN = 0, nE = 0;
  double tEnd = 0.0;
  double solverSeconds = 0.0;
  long loopIncrements = 0;
  // Explicit::explicitSolve (Explicit.C:501) overwrites Model::internalForces
  // with M^-1 f; after a run the last increment's forces are rebuilt here
  std::vector<double> fint;
  bool fintValid = false;
  std::string workdir; // where the reference writes its files
  bool vtk = false;    // result files enabled (ref_enable_vtk)
};

// Run `fn` with the working directory set to the model's (the reference
// writes its result files in the current directory).
template <typename F> void inWorkdir(RefModel *m, F fn)
{
  char cwd[4096] = "";
  const bool move = !m->workdir.empty() && getcwd(cwd, sizeof(cwd)) != nullptr && chdir(m->workdir.c_str()) == 0;
  fn();
  if (move && chdir(cwd) != 0)
    fprintf(stderr, "ref_harness: cannot return to %s\n", cwd);
}

RefModel *g_model = nullptr;
char g_err[512] = "";

void setErr(const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

/* SymTensor2 component k in the xx, xy, xz, yy, yz, zz order of its storage. */
inline double &symComp(SymTensor2 &t, int k)
{
  static const short ij[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  return t(ij[k][0], ij[k][1]);
}
} // namespace

extern "C" {

const char *ref_last_error(void) { return g_err; }

/* Build the reference model.  workdir (may be NULL) is the directory where the
 * reference writes its log file.  Returns NULL on error. */
void *ref_create(const dnl_model_desc *d, const char *workdir)
{
  if (g_model != nullptr)
  {
    setErr("only one reference model may be alive at a time");
    return nullptr;
  }
  if (d == nullptr || d->n_nodes <= 0 || d->n_elems <= 0 || d->coords == nullptr || d->conn == nullptr ||
      d->n_materials <= 0 || d->materials == nullptr)
  {
    setErr("invalid model description");
    return nullptr;
  }
  RefModel *m = new RefModel;
  m->type = d->elem_type;
  if (d->elem_type == DNL_ELQUA4NAX || d->elem_type == DNL_ELQUA4N2D)
  {
    m->npe = 4;
    m->dim = 2;
  }
  else if (d->elem_type == DNL_ELHEX8N3D)
  {
    m->npe = 8;
    m->dim = 3;
  }
  else
  {
    setErr("unknown element type %d", d->elem_type);
    delete m;
    return nullptr;
  }
  m->nN = d->n_nodes;
  m->nE = d->n_elems;
  m->tEnd = d->t_end;

  char cwd[4096] = "";
  if (workdir != nullptr)
  {
    if (getcwd(cwd, sizeof(cwd)) == nullptr)
      cwd[0] = 0;
    if (chdir(workdir) != 0)
    {
      setErr("cannot enter %s", workdir);
      delete m;
      return nullptr;
    }
  }
  // An empty DYNELA_BIN makes Settings::Settings (Settings.C:30-43) skip its
  // configuration file: the solver keeps the defaults of Solver.h, which the
  // harness overrides below.  (Unset, System::env returns a placeholder path
  // and the settings loader prints an error on every model.)  DNL_REF_SETTINGS
  // names the reference's settings directory (Sources/dnlSettings) instead,
  // for runs that write result files: their fields and title come from it.
  {
    const char *sdir = getenv("DNL_REF_SETTINGS");
    setenv("DYNELA_BIN", sdir ? sdir : "", 1);
  }
  if (workdir != nullptr)
    m->workdir = workdir;
  dynelaData = nullptr;
  m->dyn = new DynELA((char *)"ref");
  if (workdir != nullptr && cwd[0] && chdir(cwd) != 0)
    fprintf(stderr, "ref_harness: cannot return to %s\n", cwd);
  DynELA *dyn = m->dyn;

  dyn->setDefaultElement(d->elem_type == DNL_ELQUA4NAX   ? Element::ElQua4NAx
                         : d->elem_type == DNL_ELQUA4N2D ? Element::ElQua4N2D
                                                         : Element::ElHex8N3D);
  long bulkMin = 20000; // meshes from this many elements take the bulk path below
  if (const char *env = getenv("DNL_REF_BULK_MIN_ELEMS"))
    bulkMin = atol(env);
  if (m->nE < bulkMin)
  {
    // the reference's own model building (DynELA.C:168-297)
    for (long i = 0; i < m->nN; i++)
      dyn->createNode(i + 1, d->coords[3 * i], d->coords[3 * i + 1], d->coords[3 * i + 2]);
    for (long e = 0; e < m->nE; e++)
    {
      const int32_t *c = d->conn + (long)m->npe * e;
      if (m->npe == 4)
        dyn->createElement(e + 1, (long)c[0] + 1, (long)c[1] + 1, (long)c[2] + 1, (long)c[3] + 1);
      else
        dyn->createElement(e + 1, (long)c[0] + 1, (long)c[1] + 1, (long)c[2] + 1, (long)c[3] + 1, (long)c[4] + 1,
                           (long)c[5] + 1, (long)c[6] + 1, (long)c[7] + 1);
    }
  }
  else
  {
    // Large meshes: the same objects and links as DynELA::createNode /
    // createElement -> Model::add / Model::create (Model.C:67-170), with the
    // list re-indexing (ListIndex::compact, O(n) per insertion) done once at
    // the end instead of after every node and element.
    Model &model = dyn->model;
    std::vector<Node *> nodes(m->nN);
    for (long i = 0; i < m->nN; i++)
    {
      nodes[i] = new Node(i + 1, d->coords[3 * i], d->coords[3 * i + 1], d->coords[3 * i + 2]);
      model.nodes << nodes[i];
    }
    model.nodes.compact();
    for (long e = 0; e < m->nE; e++)
    {
      Element *pel = d->elem_type == DNL_ELQUA4NAX   ? (Element *)new ElQua4NAx(e + 1)
                     : d->elem_type == DNL_ELQUA4N2D ? (Element *)new ElQua4N2D(e + 1)
                                                     : (Element *)new ElHex8N3D(e + 1);
      pel->createIntegrationPoints();
      model.elements << pel;
      const int32_t *c = d->conn + (long)m->npe * e;
      for (int j = 0; j < m->npe; j++)
      {
        Node *pNode = nodes[c[j]];
        pel->addNode(pNode);
        pNode->elements << pel;
      }
    }
    model.elements.compact();
  }

  // materials: one ElementSet per material index
  for (int k = 0; k < d->n_materials; k++)
  {
    const dnl_material &mp = d->materials[k];
    JohnsonCookLaw *law = new JohnsonCookLaw();
    law->setParameters(mp.A, mp.B, mp.C, mp.n, mp.m, mp.depsp0, mp.Tm, mp.Tref);
    Material *mat = new Material((char *)"mat");
    mat->setHardeningLaw(law);
    mat->youngModulus = mp.young;
    mat->poissonRatio = mp.poisson;
    mat->density = mp.density;
    mat->heatCapacity = mp.heat_capacity;
    mat->taylorQuinney = mp.taylor_quinney;
    mat->T0 = mp.T0;
    ElementSet *es = new ElementSet((char *)"ES");
    bool any = false;
    if (d->elem_mat == nullptr)
    {
      if (k == 0)
      {
        dyn->add(es, 1, m->nE);
        any = true;
      }
    }
    else
    {
      for (long e = 0; e < m->nE; e++)
        if (d->elem_mat[e] == k)
        {
          dyn->add(es, e + 1);
          any = true;
        }
    }
    if (any)
      dyn->add(mat, es);
  }

  // time functions
  std::vector<DiscreteFunction *> funcs;
  for (int f = 0; f < d->n_functions; f++)
  {
    DiscreteFunction *df = new DiscreteFunction((char *)"F");
    for (int p = 0; p < d->functions[f].n_points; p++)
      df->add(d->functions[f].x[p], d->functions[f].y[p]);
    funcs.push_back(df);
  }

  // initial speeds: one BoundarySpeed per distinct vector
  if (d->v_init != nullptr)
  {
    std::map<std::vector<double>, NodeSet *> groups;
    for (long i = 0; i < m->nN; i++)
    {
      std::vector<double> v(d->v_init + 3 * i, d->v_init + 3 * i + 3);
      if (v[0] == 0.0 && v[1] == 0.0 && v[2] == 0.0)
        continue;
      NodeSet *&ns = groups[v];
      if (ns == nullptr)
        ns = new NodeSet((char *)"NS_init");
      dyn->add(ns, i + 1);
    }
    for (auto &g : groups)
    {
      BoundarySpeed *bs = new BoundarySpeed((char *)"BC_init");
      bs->setValue(g.first[0], g.first[1], g.first[2]);
      dyn->attachInitialBC(bs, g.second);
    }
  }

  // constant conditions: a restrain (mask) then a speed (vector, function) per node
  if (d->bc_code != nullptr)
  {
    std::map<std::vector<int>, NodeSet *> restrains;
    std::map<std::vector<double>, NodeSet *> speeds; // key: vx, vy, vz, func
    for (long i = 0; i < m->nN; i++)
    {
      std::vector<int> mask(3, 0);
      std::vector<double> sp(4, 0.0);
      bool hasR = false, hasS = false;
      sp[3] = -1;
      for (int c = 0; c < 3; c++)
      {
        int code = d->bc_code[3 * i + c];
        double val = d->bc_value ? d->bc_value[3 * i + c] : 0.0;
        int fn = d->bc_func ? d->bc_func[3 * i + c] : -1;
        if (code == DNL_BC_RESTRAIN || (code == DNL_BC_SPEED && val == 0.0))
        {
          mask[c] = 1;
          hasR = true;
        }
        else if (code == DNL_BC_SPEED)
        {
          sp[c] = val;
          if (hasS && sp[3] != (double)fn)
          {
            setErr("node %ld: one time function per node is supported by the reference", i);
            return nullptr;
          }
          sp[3] = fn;
          hasS = true;
        }
      }
      if (hasR)
      {
        NodeSet *&ns = restrains[mask];
        if (ns == nullptr)
          ns = new NodeSet((char *)"NS_restrain");
        dyn->add(ns, i + 1);
      }
      if (hasS)
      {
        NodeSet *&ns = speeds[sp];
        if (ns == nullptr)
          ns = new NodeSet((char *)"NS_speed");
        dyn->add(ns, i + 1);
      }
    }
    for (auto &g : restrains)
    {
      BoundaryRestrain *br = new BoundaryRestrain((char *)"BC_restrain");
      br->setValue(g.first[0], g.first[1], g.first[2]);
      dyn->attachConstantBC(br, g.second);
    }
    for (auto &g : speeds)
    {
      BoundarySpeed *bs = new BoundarySpeed((char *)"BC_speed");
      bs->setValue(g.first[0], g.first[1], g.first[2]);
      int fn = (int)g.first[3];
      if (fn >= 0)
      {
        if (fn >= (int)funcs.size())
        {
          setErr("function index %d out of range", fn);
          return nullptr;
        }
        bs->setFunction(funcs[fn]);
      }
      dyn->attachConstantBC(bs, g.second);
    }
  }

  Explicit *s = new Explicit((char *)"Solver");
  s->setTimes(d->t_start, d->t_end);
  dyn->add(s);
  s->setTimeStepMethod(d->ts_method == DNL_TS_POWER_ITERATION ? Solver::PowerIteration : Solver::Courant);
  s->setComputeTimeStepFrequency(d->ts_freq > 0 ? d->ts_freq : 10);
  s->setTimeStepSafetyFactor(d->ts_safety > 0 ? d->ts_safety : 0.9);
  if (d->rho_b >= 0.0 && d->rho_b <= 1.0)
    s->setDissipation(d->rho_b);
  s->_reportFrequency = 1 << 30; // keep stdout quiet
  // DynELA::setStressComputation (DynELA.C:1407-1431)
  if (d->stress_method == DNL_STRESS_DIRECT)
    dyn->setStressComputation((char *)"Direct");
  m->solver = s;
  g_model = m;
  return m;
}

void ref_set_threads(int n)
{
  if (g_model != nullptr && n > 0)
    g_model->dyn->parallel.setCores(n);
}

/* Model::initSolve + the pre-loop part of Explicit::solve (Explicit.C:143-181). */
int ref_init(void *h)
{
  RefModel *m = (RefModel *)h;
  if (m == nullptr || m != g_model)
    return DNL_ERR_ARG;
  DynELA *dyn = m->dyn;
  Model &model = dyn->model;
  dyn->initSolve();
  Explicit *s = m->solver;
  s->_solveUpToTime = m->tEnd;
  model.computeJacobian(true);
  model.computeUnderJacobian(true);
  model.computeMassMatrix();
  s->computeTimeStep(true);
  model.computeStrains();
  model.computePressure();
  model.computeStress(s->timeStep);
  model.computeFinalRotation();
  model.computeInternalForces();
  return DNL_OK;
}

/* Run the increment loop of Explicit::solve (Explicit.C:184-256, the same calls
 * in the same order) until currentTime reaches min(t_stop, end time) or
 * max_incs increments have run.  Returns the number of increments run. */
long ref_run(void *h, double t_stop, long max_incs)
{
  RefModel *m = (RefModel *)h;
  if (m == nullptr || m != g_model)
    return -1;
  Model *model = &m->dyn->model;
  Explicit *s = m->solver;
  double upTo = s->_solveUpToTime;
  long k = 0;
  char cwd[4096] = "";
  const bool moved = m->vtk && getcwd(cwd, sizeof(cwd)) != nullptr && chdir(m->workdir.c_str()) == 0;
  auto t0 = std::chrono::steady_clock::now();
  m->dyn->cpuTimes.timer("Solver")->start();
  while (model->currentTime < upTo && model->currentTime < t_stop && (max_incs <= 0 || k < max_incs))
  {
    s->updateTimes();
    s->computePredictions();
    model->computeStrains();
    model->computePressure();
    model->computeStress(s->timeStep);
    model->computeFinalRotation();
    model->computeInternalForces();
    s->explicitSolve();
    s->computeDensity();
    s->endStep();
    if (model->currentTime < upTo)
    {
      model->computeJacobian();
      model->computeUnderJacobian();
      s->computeTimeStep();
    }
    k++;
  }
  m->dyn->cpuTimes.timer("Solver")->stop();
  m->solverSeconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  m->loopIncrements += k;
  if (moved && chdir(cwd) != 0)
    fprintf(stderr, "ref_harness: cannot return to %s\n", cwd);
  if (k > 0)
  {
    // internal forces of the last increment: M (M^-1 f), outside the timing
    const long n = (long)m->nN * m->dim;
    m->fint.resize(n);
    for (long i = 0; i < n; i++)
      m->fint[i] = model->internalForces(i) * model->massMatrix(i);
    m->fintValid = true;
  }
  return k;
}

/* The reference's own result files: save times set (DynELA::setSaveTimes,
 * DynELA.C:479-487) and the initial file written now, as DynELA::solve does
 * after initSolve (DynELA.C:745, writeResultFile, DynELA.C:489-504); the
 * reference's Explicit::endStep then writes the files of the save times
 * during ref_run (Explicit.C:548), as <workdir>/<model name>NNN.vtk with the
 * fields of its settings (VtkInterface::initFields, VtkInterface.C:224-242;
 * see DNL_REF_SETTINGS in ref_create). */
int ref_enable_vtk(void *h, double start, double end, double inc)
{
  RefModel *m = (RefModel *)h;
  if (m == nullptr || m != g_model || m->workdir.empty())
    return DNL_ERR_ARG;
  m->dyn->setSaveTimes(start, end, inc);
  m->vtk = true;
  inWorkdir(m, [&] { m->dyn->writeResultFile(); });
  return DNL_OK;
}

/* The last result file of DynELA::solve (DynELA.C:770, writeVTKFile). */
int ref_write_final_vtk(void *h)
{
  RefModel *m = (RefModel *)h;
  if (m == nullptr || m != g_model || !m->vtk)
    return DNL_ERR_ARG;
  inWorkdir(m, [&] { m->dyn->writeVTKFile(); });
  return DNL_OK;
}

/* The reference's own Explicit::solve(upTo) (pre-loop part + loop), used to pin
 * ref_init + ref_run against it. */
int ref_solve_native(void *h)
{
  RefModel *m = (RefModel *)h;
  if (m == nullptr || m != g_model)
    return DNL_ERR_ARG;
  m->dyn->initSolve();
  m->solver->solve(m->tEnd);
  return DNL_OK;
}

double ref_solver_seconds(void *h) { return h ? ((RefModel *)h)->solverSeconds : -1.0; }

/* time, timeStep, increment */
void ref_control(void *h, double *out3)
{
  RefModel *m = (RefModel *)h;
  out3[0] = m->dyn->model.currentTime;
  out3[1] = m->solver->timeStep;
  out3[2] = (double)m->solver->currentIncrement;
}

/* Nodal field (DNL_NODE_*) as [nN*3]. */
int ref_get_nodes(void *h, int field, double *out)
{
  RefModel *m = (RefModel *)h;
  if (m == nullptr || m != g_model)
    return DNL_ERR_ARG;
  Model &model = m->dyn->model;
  for (long i = 0; i < m->nN; i++)
  {
    Node *n = model.nodes(i);
    for (int c = 0; c < 3; c++)
    {
      double v = 0.0;
      switch (field)
      {
      case DNL_NODE_COORDS: v = n->coords(c); break;
      case DNL_NODE_DISP: v = n->disp(c); break;
      case DNL_NODE_U: v = n->field0->u(c); break;
      case DNL_NODE_SPEED: v = n->field0->speed(c); break;
      case DNL_NODE_ACCEL: v = n->field0->acceleration(c); break;
      case DNL_NODE_MASS: v = n->mass; break;
      case DNL_NODE_FORCE:
        v = (c >= m->dim) ? 0.0 : m->fintValid ? m->fint[i * m->dim + c] : model.internalForces(i * m->dim + c);
        break;
      case DNL_NODE_SPEED_PREV: v = n->field1->speed(c); break;
      case DNL_NODE_U_PREV: v = n->field1->u(c); break;
      case DNL_NODE_ACCEL_PREV: v = n->field1->acceleration(c); break;
      default: return DNL_ERR_ARG;
      }
      out[3 * i + c] = v;
    }
  }
  return DNL_OK;
}

int ref_set_nodes(void *h, int field, const double *in)
{
  RefModel *m = (RefModel *)h;
  if (m == nullptr || m != g_model)
    return DNL_ERR_ARG;
  Model &model = m->dyn->model;
  for (long i = 0; i < m->nN; i++)
  {
    Node *n = model.nodes(i);
    for (int c = 0; c < 3; c++)
    {
      double v = in[3 * i + c];
      switch (field)
      {
      case DNL_NODE_COORDS: n->coords(c) = v; break;
      case DNL_NODE_DISP: n->disp(c) = v; break;
      case DNL_NODE_U: n->field0->u(c) = v; break;
      case DNL_NODE_SPEED: n->field0->speed(c) = v; break;
      case DNL_NODE_ACCEL: n->field0->acceleration(c) = v; break;
      default: return DNL_ERR_ARG;
      }
    }
  }
  return DNL_OK;
}

static double *ipField(IntegrationPoint *ip, int comp)
{
  if (comp < 6) return &symComp(ip->Stress, comp);
  if (comp < 12) return &symComp(ip->Strain, comp - 6);
  if (comp < 18) return &symComp(ip->PlasticStrain, comp - 12);
  switch (comp)
  {
  case DNL_IP_EPSP: return &ip->plasticStrain;
  case DNL_IP_DEPSP: return &ip->plasticStrainRate;
  case DNL_IP_GAMMA: return &ip->gamma;
  case DNL_IP_GAMMA_CUM: return &ip->gammaCumulate;
  case DNL_IP_YIELD: return &ip->yieldStress;
  case DNL_IP_T: return &ip->T;
  case DNL_IP_PRESSURE: return &ip->pressure;
  case DNL_IP_EINT: return &ip->internalEnergy;
  case DNL_IP_EINEL: return &ip->inelasticEnergy;
  case DNL_IP_DENSITY: return &ip->density;
  case DNL_IP_DETJ0: return &ip->detJ0;
  }
  return nullptr;
}

/* Integration-point state [DNL_IP_NCOMP * nIP], component-major. */
int ref_get_ips(void *h, double *out)
{
  RefModel *m = (RefModel *)h;
  if (m == nullptr || m != g_model)
    return DNL_ERR_ARG;
  long nIP = m->nE * m->npe;
  for (long e = 0; e < m->nE; e++)
  {
    Element *el = m->dyn->model.elements(e);
    for (int g = 0; g < m->npe; g++)
    {
      IntegrationPoint *ip = el->integrationPoints(g);
      for (int c = 0; c < DNL_IP_NCOMP; c++)
        out[(long)c * nIP + e * m->npe + g] = *ipField(ip, c);
    }
  }
  return DNL_OK;
}

/* Intermediate values of one integration point after the last element pass,
 * for inspection: StrainInc (6, SymTensor2 order) then R (9, row-major). */
int ref_point_kinematics(void *h, long q, double *out15)
{
  RefModel *m = (RefModel *)h;
  if (m == nullptr || m != g_model || q < 0 || q >= m->nE * m->npe)
    return DNL_ERR_ARG;
  IntegrationPoint *ip = m->dyn->model.elements(q / m->npe)->integrationPoints(q % m->npe);
  for (int k = 0; k < 6; k++)
    out15[k] = symComp(ip->StrainInc, k);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      out15[6 + 3 * i + j] = ip->R(i, j);
  return DNL_OK;
}

/* The largest departure from orthogonality, max |R^T R - I|, of the rotation
 * of every integration point after the last element pass (Tensor2::
 * polarCuppenLnU, Tensor2.C:1442-1457); out2 = {value, point}. */
int ref_rotation_orthogonality(void *h, double *out2)
{
  RefModel *m = (RefModel *)h;
  if (m == nullptr || m != g_model)
    return DNL_ERR_ARG;
  double worst = 0.0;
  long at = -1;
  for (long e = 0; e < m->nE; e++)
    for (int g = 0; g < m->npe; g++)
    {
      const Tensor2 &R = m->dyn->model.elements(e)->integrationPoints(g)->R;
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
        {
          double s = (i == j) ? -1.0 : 0.0;
          for (int k = 0; k < 3; k++)
            s += R(k, i) * R(k, j);
          if (fabs(s) > worst)
          {
            worst = fabs(s);
            at = e * m->npe + g;
          }
        }
    }
  out2[0] = worst;
  out2[1] = (double)at;
  return DNL_OK;
}

int ref_set_ips(void *h, const double *in)
{
  RefModel *m = (RefModel *)h;
  if (m == nullptr || m != g_model)
    return DNL_ERR_ARG;
  long nIP = m->nE * m->npe;
  for (long e = 0; e < m->nE; e++)
  {
    Element *el = m->dyn->model.elements(e);
    for (int g = 0; g < m->npe; g++)
    {
      IntegrationPoint *ip = el->integrationPoints(g);
      for (int c = 0; c < DNL_IP_NCOMP; c++)
        *ipField(ip, c) = in[(long)c * nIP + e * m->npe + g];
    }
  }
  return DNL_OK;
}

/* One element pass on the current state (Explicit.C:204-226 after a Jacobian
 * of the current coordinates, Model.C:754-774): strains, pressure, stress,
 * final rotation, internal forces, then the density of Explicit::computeDensity
 * (Explicit.C:555-562).  Forces land in DNL_NODE_FORCE. */
int ref_element_pass(void *h, double timeStep)
{
  RefModel *m = (RefModel *)h;
  if (m == nullptr || m != g_model)
    return DNL_ERR_ARG;
  Model &model = m->dyn->model;
  m->solver->timeStep = timeStep;
  model.computeJacobian();
  model.computeStrains();
  model.computePressure();
  model.computeStress(timeStep);
  model.computeFinalRotation();
  model.computeInternalForces();
  m->fintValid = false; // Model::internalForces holds f itself
  m->solver->computeDensity();
  return DNL_OK;
}

/* Courant critical time step min_e l_e / c_e (Model.C:636-669) on the current state. */
double ref_courant(void *h)
{
  RefModel *m = (RefModel *)h;
  return m->dyn->model.computeCourantTimeStep();
}

/* Per-element characteristic length and wave speed. */
int ref_element_lengths(void *h, double *len, double *wave)
{
  RefModel *m = (RefModel *)h;
  if (m == nullptr || m != g_model)
    return DNL_ERR_ARG;
  for (long e = 0; e < m->nE; e++)
  {
    Element *el = m->dyn->model.elements(e);
    len[e] = el->getCharacteristicLength();
    wave[e] = el->getElongationWaveSpeed();
  }
  return DNL_OK;
}

/* Per-phase wall time of the reference's Timers ("Strains", "Stress", ...). */
double ref_timer(void *h, const char *name)
{
  RefModel *m = (RefModel *)h;
  if (m == nullptr)
    return -1.0;
  return m->dyn->cpuTimes.timer(name)->getTotal();
}

/* Release the handle.  The reference objects are leaked on purpose: the
 * reference frees nothing it allocates and its destructor writes report files. */
void ref_destroy(void *h)
{
  RefModel *m = (RefModel *)h;
  if (m == nullptr || m != g_model)
    return;
  dynelaData = nullptr;
  g_model = nullptr;
  delete m;
}

} // extern "C"
