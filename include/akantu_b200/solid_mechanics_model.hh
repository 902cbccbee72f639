/*
 * akantu_b200/solid_mechanics_model.hh -- C++ drop-in API of the explicit
 * lumped-mass step, header-only over the C ABI (akb_capi.h, libakb.so).
 *
 * Mirrors the reference surface used by explicit drivers
 * (src/model/solid_mechanics/solid_mechanics_model.hh:61-321,
 *  src/model/model.hh:74-131, src/mesh/mesh.hh:121-281,
 *  src/io/parser/parser.hh:344-432, src/common/aka_common.hh:48,662):
 *
 *   initialize("material.dat", argc, argv);
 *   Mesh mesh(3); mesh.read("bar.msh");
 *   SolidMechanicsModel model(mesh);
 *   model.initFull(_analysis_method = _explicit_lumped_mass);
 *   model.setTimeStep(0.8 * model.getStableTimeStep());
 *   Array<Real> & u = model.getDisplacement();   // host view, edit in place
 *   for (...) model.solveStep();
 *
 * The nodal arrays live on the GPU.  The getters return host arrays that
 * the model refreshes after a step and uploads again before the next step
 * when the caller may have changed them (any non-const getter call marks the
 * array), which gives the reference's "edit the array between steps"
 * semantics.  Errors throw akantu_b200::Exception with the library message.
 */
#ifndef AKANTU_B200_SOLID_MECHANICS_MODEL_HH_
#define AKANTU_B200_SOLID_MECHANICS_MODEL_HH_

#include <cstdint>
#include <deque>
#include <fstream>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../akb_capi.h"

namespace akantu_b200 {

using Real = double;
using Int = int64_t;
using Idx = int32_t;
using ID = std::string;

class Exception : public std::runtime_error {
public:
  Exception(int code, const std::string &msg) : std::runtime_error(msg), code_(code) {}
  int code() const { return code_; }

private:
  int code_;
};

inline void check(int rc) {
  if (rc != AKB_OK) throw Exception(rc, akb_last_error());
}

/* ---- element types, analysis method, axes -------------------------------- */
enum ElementType {
  _tetrahedron_4 = AKB_TETRAHEDRON_4,
  _hexahedron_8 = AKB_HEXAHEDRON_8,
  _triangle_6 = AKB_TRIANGLE_6,
  _not_defined = -1
};
enum AnalysisMethod { _explicit_lumped_mass = AKB_EXPLICIT_LUMPED_MASS };
enum SpatialDirection { _x = 0, _y = 1, _z = 2 };
constexpr Int _all_dimensions = -1;

// named argument of initFull: model.initFull(_analysis_method = _explicit_lumped_mass)
struct AnalysisMethodArg {
  AnalysisMethod method;
  int precision;
};
struct AnalysisMethodTag {
  AnalysisMethodArg operator=(AnalysisMethod m) const { return {m, AKB_PRECISION_FP64}; }
};
inline constexpr AnalysisMethodTag _analysis_method{};

/* ---- Array: row-major tuples (size x nb_component), src/common/aka_array.hh */
template <class T> class Array {
public:
  Array(Int size = 0, Int nb_component = 1, T value = T())
      : n_(size), c_(nb_component), v_(allocate(size * nb_component)) {
    set(value);
  }
  Array(const Array &o) : n_(o.n_), c_(o.c_), v_(allocate(o.n_ * o.c_)) {
    for (Int k = 0; k < n_ * c_; ++k) v_[k] = o.v_[k];
  }
  Array(Array &&) = default;
  Array &operator=(const Array &o) {
    if (this != &o) {
      Array tmp(o);
      *this = std::move(tmp);
    }
    return *this;
  }
  Array &operator=(Array &&) = default;
  Int size() const { return n_; }
  Int getNbComponent() const { return c_; }
  T &operator()(Int i, Int c = 0) { return v_[i * c_ + c]; }
  const T &operator()(Int i, Int c = 0) const { return v_[i * c_ + c]; }
  T *data() { return v_.get(); }
  const T *data() const { return v_.get(); }
  void resize(Int size) {
    std::unique_ptr<T[]> nv = allocate(size * c_);
    for (Int k = 0; k < std::min(size, n_) * c_; ++k) nv[k] = v_[k];
    v_ = std::move(nv);
    n_ = size;
  }
  void set(T value) {
    for (Int k = 0; k < n_ * c_; ++k) v_[k] = value;
  }
  void zero() { set(T()); }

private:
  // never a zero-length allocation, so data() is always a valid pointer
  static std::unique_ptr<T[]> allocate(Int n) { return std::unique_ptr<T[]>(new T[n > 0 ? n : 1]()); }
  Int n_, c_;
  std::unique_ptr<T[]> v_;
};

/* ---- static parser (getStaticParser().parse / initialize) --------------- */
class Parser {
public:
  void parse(const std::string &path) {
    std::ifstream f(path);
    if (!f) throw Exception(AKB_EIO, "cannot open " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    texts_.push_back(ss.str());
  }
  void parseText(const std::string &text) { texts_.push_back(text); }
  void clear() { texts_.clear(); }
  const std::vector<std::string> &texts() const { return texts_; }

private:
  std::vector<std::string> texts_;
};

inline Parser &getStaticParser() {
  static Parser parser;
  return parser;
}

inline void initialize(const std::string &input_file, int /*argc*/ = 0, char ** /*argv*/ = nullptr) {
  if (!input_file.empty()) getStaticParser().parse(input_file);
}

/* ---- Mesh ------------------------------------------------------------------ */
class Mesh {
public:
  explicit Mesh(Int spatial_dimension) : dim_(spatial_dimension), nodes_(0, spatial_dimension) {}

  // Mesh::read for gmsh 2.x and 4.x ASCII files: the elements of the type
  // matching the dimension (_triangle_6 in 2D; _hexahedron_8, else
  // _tetrahedron_4 in 3D); the file's physical groups become node groups
  void read(const std::string &path, ElementType type = _not_defined) {
    std::vector<ElementType> types;
    if (type != _not_defined) types = {type};
    else if (dim_ == 2) types = {_triangle_6};
    else types = {_hexahedron_8, _tetrahedron_4};
    for (ElementType t : types) {
      akb_mesh *m = nullptr;
      check(akb_mesh_read_msh(path.c_str(), (int)dim_, t, &m));
      int64_t nn = 0, ne = 0;
      int npe = 0;
      check(akb_mesh_sizes(m, &nn, &ne, &npe));
      if (ne == 0 && types.size() > 1 && t != types.back()) {
        akb_mesh_free(m);
        continue;
      }
      nodes_ = Array<Real>(nn, dim_);
      conn_ = Array<Idx>(ne, npe);
      tags_ = Array<Idx>(ne, 1);
      check(akb_mesh_copy(m, nodes_.data(), conn_.data(), tags_.data()));
      int ng = 0;
      check(akb_mesh_nb_groups(m, &ng));
      for (int k = 0; k < ng; ++k) {
        char name[256];
        int64_t count = 0;
        check(akb_mesh_group(m, k, name, sizeof(name), nullptr, &count, nullptr));
        std::vector<int32_t> members((size_t)count);
        check(akb_mesh_group(m, k, nullptr, 0, nullptr, nullptr, members.data()));
        groups_[name] = std::set<Idx>(members.begin(), members.end());
      }
      int nb_names = 0;
      check(akb_mesh_nb_element_names(m, &nb_names));
      has_physical_names_ = nb_names >= 0;
      physical_names_.clear();
      if (has_physical_names_ && ne > 0) {
        std::vector<std::string> table((size_t)nb_names);
        for (int k = 0; k < nb_names; ++k) {
          char name[256];
          check(akb_mesh_element_names(m, k, name, sizeof(name), nullptr));
          table[k] = name;
        }
        std::vector<int32_t> index((size_t)ne);
        check(akb_mesh_element_names(m, 0, nullptr, 0, index.data()));
        for (int32_t i : index) physical_names_.push_back(table[i]);
      }
      akb_mesh_free(m);
      type_ = t;
      return;
    }
  }

  void setElements(ElementType type, const Array<Real> &nodes, const Array<Idx> &conn) {
    type_ = type;
    nodes_ = nodes;
    conn_ = conn;
    tags_ = Array<Idx>(conn.size(), 1);
  }

  Int getSpatialDimension() const { return dim_; }
  Int getNbNodes() const { return nodes_.size(); }
  Int getNbElement(ElementType = _not_defined) const { return conn_.size(); }
  ElementType getElementType() const { return type_; }
  Array<Real> &getNodes() { return nodes_; }
  const Array<Real> &getNodes() const { return nodes_; }
  const Array<Idx> &getConnectivity(ElementType = _not_defined) const { return conn_; }
  const Array<Idx> &getPhysicalTags() const { return tags_; }

  // element data read from the file (Mesh::getData): "physical_names"
  // (std::string, each element's physical name) and "tag_0" (Idx, its first
  // physical tag)
  template <typename T> std::vector<T> getData(const ID &name, ElementType = _not_defined) const {
    if constexpr (std::is_same_v<T, std::string>) {
      if (name != "physical_names" || !has_physical_names_)
        throw Exception(AKB_EINVAL, "the mesh has no element data " + name);
      return physical_names_;
    } else {
      if (name != "tag_0") throw Exception(AKB_EINVAL, "the mesh has no element data " + name);
      return std::vector<T>(tags_.data(), tags_.data() + tags_.size());
    }
  }

  // named node groups (src/mesh/group_manager.hh), used by applyBC
  void createNodeGroup(const ID &name, const std::vector<Idx> &nodes) {
    groups_[name] = std::set<Idx>(nodes.begin(), nodes.end());
  }
  const std::set<Idx> &getNodeGroup(const ID &name) const { return groups_.at(name); }

private:
  Int dim_;
  ElementType type_ = _not_defined;
  Array<Real> nodes_;
  Array<Idx> conn_{0, 4}, tags_{0, 1};
  std::map<ID, std::set<Idx>> groups_;
  bool has_physical_names_ = false;
  std::vector<std::string> physical_names_;
};

namespace BC {
namespace Dirichlet {
// BC::Dirichlet::FixedValue(value, axis)
// (boundary_condition_functor_inline_impl.hh:53-61)
struct FixedValue {
  FixedValue(Real v, SpatialDirection ax = _x) : value(v), axis(ax) {}
  Real value;
  SpatialDirection axis;
};
}  // namespace Dirichlet
namespace Neumann {
// BC::Neumann::FromHigherDim(stress): traction stress . n on the group's
// boundary facets, added to the external force (boundary_condition_tmpl.hh:100-164)
struct FromHigherDim {
  explicit FromHigherDim(const Array<Real> &stress_dim_x_dim) : stress(stress_dim_x_dim) {}
  Array<Real> stress;  // (i, j) = stress_ij
};
}  // namespace Neumann
}  // namespace BC

class SolidMechanicsModel;

/* ---- material selection (src/model/common/constitutive_laws/
 * constitutive_law_selector.hh:45-150) ----------------------------------------- */
struct Element {
  ElementType type = _not_defined;
  Idx element = 0;
};

class MaterialSelector : public std::enable_shared_from_this<MaterialSelector> {
public:
  virtual ~MaterialSelector() = default;
  virtual Idx operator()(const Element &element) {
    return fallback_selector_ ? (*fallback_selector_)(element) : fallback_value_;
  }
  void setFallback(Idx f) { fallback_value_ = f; }
  void setFallback(const std::shared_ptr<MaterialSelector> &f) { fallback_selector_ = f; }
  Idx getFallbackValue() const { return fallback_value_; }

private:
  Idx fallback_value_ = 0;
  std::shared_ptr<MaterialSelector> fallback_selector_;
};

// a string datum is the name of the element's material (an element whose
// name names no material takes the fallback), an integer datum its index
template <typename T> class ElementDataMaterialSelector : public MaterialSelector {
public:
  ElementDataMaterialSelector(std::vector<T> data, SolidMechanicsModel &model, Idx first_index = 1)
      : data_(std::move(data)), model_(&model), first_index_(first_index) {}
  inline Idx operator()(const Element &element) override;
  Idx getFirstIndex() const { return first_index_; }

private:
  std::vector<T> data_;
  SolidMechanicsModel *model_;
  Idx first_index_;
};

template <typename T> class MeshDataMaterialSelector : public ElementDataMaterialSelector<T> {
public:
  inline MeshDataMaterialSelector(const ID &name, SolidMechanicsModel &model, Idx first_index = 1);
};

/* ---- Material view ---------------------------------------------------------- */
class Material {
public:
  Material(SolidMechanicsModel &model, int index) : model_(&model), index_(index) {}
  inline Real get(const ID &param) const;
  Real getRho() const { return get("rho"); }
  inline ID getName() const;
  // the mesh elements that this material holds
  inline Array<Idx> getElementFilter(ElementType = _not_defined) const;
  // quadrature-point internals, material-local element order, [nq][dim*dim]
  inline Array<Real> getStress(ElementType = _not_defined);
  inline Array<Real> getGradU(ElementType = _not_defined);
  inline Array<Real> getInternal(const ID &name, ElementType = _not_defined);
  // writes an internal in the getter's layout (only "eigen_grad_u"); the
  // reference assigns getInternal<Real>(name)(type) in place
  inline void setInternal(const ID &name, const Array<Real> &values,
                          ElementType = _not_defined);

private:
  inline Array<Real> qp(int field);
  static inline int internalId(const ID &name);
  SolidMechanicsModel *model_;
  int index_;
};

/* ---- SolidMechanicsModel ------------------------------------------------- */
class SolidMechanicsModel {
public:
  explicit SolidMechanicsModel(Mesh &mesh, Int dim = _all_dimensions,
                               const ID &id = "solid_mechanics_model")
      : mesh_(mesh), dim_(dim == _all_dimensions ? mesh.getSpatialDimension() : dim), id_(id) {
    check(akb_model_create((int)dim_, mesh.getElementType(), mesh.getNodes().data(),
                           mesh.getNbNodes(), mesh.getConnectivity().data(),
                           mesh.getNbElement(), &h_));
  }
  ~SolidMechanicsModel() {
    if (h_) akb_model_destroy(h_);
  }
  SolidMechanicsModel(const SolidMechanicsModel &) = delete;
  SolidMechanicsModel &operator=(const SolidMechanicsModel &) = delete;

  void initFull(AnalysisMethodArg arg = {_explicit_lumped_mass, AKB_PRECISION_FP64}) {
    for (const auto &text : getStaticParser().texts())
      check(akb_model_load_materials(h_, text.c_str()));
    applySelector();
    check(akb_model_init_full(h_, arg.method, arg.precision));
  }

  // element -> material index, before initFull
  void setElementMaterials(const std::vector<Idx> &material_of_element) {
    check(akb_model_set_element_materials(h_, material_of_element.data()));
    element_materials_ = material_of_element;
  }
  // applied by initFull, once the materials are known
  void setMaterialSelector(std::shared_ptr<MaterialSelector> selector) {
    selector_ = std::move(selector);
  }
  MaterialSelector *getMaterialSelector() { return selector_.get(); }
  // material index of a name, -1 when no material has that name
  Int getMaterialIndex(const ID &name) {
    for (Int i = 0; i < getNbMaterials(); ++i)
      if (getMaterial(i).getName() == name) return i;
    return -1;
  }
  const std::vector<Idx> &getElementMaterials() {
    if (element_materials_.size() != (size_t)mesh_.getNbElement())
      element_materials_.assign((size_t)mesh_.getNbElement(), 0);
    return element_materials_;
  }
  // FP32 element math with FP64 nodal state (see akb_precision)
  void initFullMixedPrecision() { check(akb_model_load_and_init_mixed()); }

  Real getStableTimeStep() {
    syncUp();
    Real dt = 0;
    check(akb_model_get_stable_time_step(h_, &dt));
    return dt;
  }
  void setTimeStep(Real dt, const ID & = "") { check(akb_model_set_time_step(h_, dt)); }
  Real getTimeStep(const ID & = "") const {
    Real dt = 0;
    check(akb_model_get_time_step(h_, &dt));
    return dt;
  }

  // ModelSolver::solveStep; nsteps > 1 enqueues several steps at once
  void solveStep(const ID & = "", Int nsteps = 1) {
    syncUp();
    check(akb_model_solve_step(h_, nsteps));
    mirrors_.clear();
    blocked_.reset();
  }

  Array<Real> &getDisplacement() { return nodal(AKB_DISPLACEMENT, true); }
  Array<Real> &getVelocity() { return nodal(AKB_VELOCITY, true); }
  Array<Real> &getAcceleration() { return nodal(AKB_ACCELERATION, true); }
  Array<Real> &getExternalForce() { return nodal(AKB_EXTERNAL_FORCE, true); }
  const Array<Real> &getInternalForce() {
    syncUp();
    return nodal(AKB_INTERNAL_FORCE, false);
  }
  const Array<Real> &getMass() { return nodal(AKB_MASS, false); }
  // SolidMechanicsModel::getPreviousDisplacement / getIncrement
  // (solid_mechanics_model.hh:284-293): kept while increment tracking is on
  void setIncrementTracking(bool on = true) {
    syncUp();
    check(akb_model_set_increment_tracking(h_, on ? 1 : 0));
    mirrors_.erase(AKB_PREVIOUS_DISPLACEMENT);
    mirrors_.erase(AKB_DISPLACEMENT_INCREMENT);
  }
  const Array<Real> &getPreviousDisplacement() {
    syncUp();
    return nodal(AKB_PREVIOUS_DISPLACEMENT, false);
  }
  const Array<Real> &getIncrement() {
    syncUp();
    return nodal(AKB_DISPLACEMENT_INCREMENT, false);
  }
  const Array<Real> &getCurrentPosition() {
    syncUp();
    mirrors_.erase(AKB_CURRENT_POSITION);
    return nodal(AKB_CURRENT_POSITION, false);
  }
  Array<bool> &getBlockedDOFs() {
    if (!blocked_) {
      std::vector<uint8_t> raw(mesh_.getNbNodes() * dim_);
      check(akb_model_get_nodal(h_, AKB_BLOCKED_DOFS, raw.data(), (int64_t)raw.size()));
      blocked_ = std::make_unique<Array<bool>>(mesh_.getNbNodes(), dim_);
      for (size_t k = 0; k < raw.size(); ++k) blocked_->data()[k] = raw[k] != 0;
    }
    blocked_dirty_ = true;
    return *blocked_;
  }

  // applyBC(BC::Dirichlet::FixedValue(v, axis), group)
  void applyBC(const BC::Dirichlet::FixedValue &bc, const ID &group) {
    auto &blocked = getBlockedDOFs();
    auto &u = getDisplacement();
    for (Idx n : mesh_.getNodeGroup(group)) {
      blocked(n, bc.axis) = true;
      u(n, bc.axis) = bc.value;
    }
  }

  // applyBC(BC::Neumann::FromHigherDim(stress), group)
  void applyBC(const BC::Neumann::FromHigherDim &bc, const ID &group) {
    syncUp();
    std::vector<int32_t> nodes(mesh_.getNodeGroup(group).begin(), mesh_.getNodeGroup(group).end());
    std::vector<Real> sig((size_t)dim_ * dim_);
    for (Int i = 0; i < dim_; ++i)
      for (Int j = 0; j < dim_; ++j) sig[i + dim_ * j] = bc.stress(i, j);  // column-major
    check(akb_model_apply_neumann_stress(h_, nodes.data(), (int64_t)nodes.size(), sig.data()));
    mirrors_.erase(AKB_EXTERNAL_FORCE);
  }

  void assembleInternalForces() {
    syncUp();
    check(akb_model_assemble_internal_forces(h_));
    mirrors_.erase(AKB_INTERNAL_FORCE);
  }

  // the imposed-displacement loop of a driver done on the device: `axis` of
  // the group's nodes is blocked and, before every later step k, moved to
  // u_now + sum_{j<=k} dt v_max min(1, j / ramp_steps)
  void setPrescribedVelocityRamp(const ID &group, Int axis, Real v_max, Int ramp_steps) {
    syncUp();
    std::vector<int64_t> dofs;
    for (Idx n : mesh_.getNodeGroup(group)) dofs.push_back((int64_t)n * dim_ + axis);
    check(akb_model_set_prescribed_velocity_ramp(h_, dofs.data(), (int64_t)dofs.size(), v_max,
                                                 ramp_steps));
    blocked_.reset();
    blocked_dirty_ = false;
  }

  // fastest launch shapes on the current state (results unchanged)
  void autotune(int repeats = 5) {
    syncUp();
    check(akb_model_autotune(h_, repeats));
  }

  Real getEnergy(const ID &energy_id) {
    syncUp();
    Real e = 0;
    check(akb_model_get_energy(h_, energy_id.c_str(), &e));
    return e;
  }

  Int getNbMaterials() const {
    int n = 0;
    check(akb_model_nb_materials(h_, &n));
    return n;
  }
  Material &getMaterial(Int i) {
    while ((Int)materials_.size() <= i) materials_.emplace_back(*this, (int)materials_.size());
    return materials_[i];
  }
  Material &getMaterial(const ID &name) {
    const Int i = getMaterialIndex(name);
    if (i < 0) throw Exception(AKB_EMATERIAL, "no material named " + name);
    return getMaterial(i);
  }

  Int getSpatialDimension() const { return dim_; }
  Mesh &getMesh() { return mesh_; }
  akb_model *handle() { return h_; }

  // uploads the host arrays handed out since the last step
  void syncUp() {
    for (int f : handed_out_) {
      auto &a = mirrors_.at(f);
      check(akb_model_set_nodal(h_, f, a.data(), (int64_t)(a.size() * dim_ * sizeof(Real))));
    }
    handed_out_.clear();
    if (blocked_dirty_ && blocked_) {
      std::vector<uint8_t> raw(blocked_->size() * dim_);
      for (size_t k = 0; k < raw.size(); ++k) raw[k] = blocked_->data()[k] ? 1 : 0;
      check(akb_model_set_nodal(h_, AKB_BLOCKED_DOFS, raw.data(), (int64_t)raw.size()));
    }
    blocked_dirty_ = false;
  }

private:
  int akb_model_load_and_init_mixed() {
    for (const auto &text : getStaticParser().texts()) {
      int rc = akb_model_load_materials(h_, text.c_str());
      if (rc != AKB_OK) return rc;
    }
    applySelector();
    return akb_model_init_full(h_, AKB_EXPLICIT_LUMPED_MASS, AKB_PRECISION_MIXED);
  }

  void applySelector() {
    if (!selector_) return;
    std::vector<Idx> mat((size_t)mesh_.getNbElement());
    for (size_t e = 0; e < mat.size(); ++e) mat[e] = (*selector_)(Element{mesh_.getElementType(), (Idx)e});
    setElementMaterials(mat);
  }

  Array<Real> &nodal(int field, bool writable) {
    auto it = mirrors_.find(field);
    if (it == mirrors_.end()) {
      Array<Real> a(mesh_.getNbNodes(), dim_);
      check(akb_model_get_nodal(h_, field, a.data(), (int64_t)(a.size() * dim_ * sizeof(Real))));
      it = mirrors_.emplace(field, std::move(a)).first;
    }
    if (writable) handed_out_.insert(field);
    return it->second;
  }

  Mesh &mesh_;
  Int dim_;
  ID id_;
  akb_model *h_ = nullptr;
  std::map<int, Array<Real>> mirrors_;
  std::set<int> handed_out_;
  std::unique_ptr<Array<bool>> blocked_;
  bool blocked_dirty_ = false;
  std::deque<Material> materials_;  // references stay valid as it grows
  std::shared_ptr<MaterialSelector> selector_;
  std::vector<Idx> element_materials_;
};

template <typename T> Idx ElementDataMaterialSelector<T>::operator()(const Element &element) {
  if (element.element < 0 || (size_t)element.element >= data_.size())
    return MaterialSelector::operator()(element);
  if constexpr (std::is_same_v<T, std::string>) {
    const Int i = model_->getMaterialIndex(data_[element.element]);
    return i >= 0 ? (Idx)i : MaterialSelector::operator()(element);
  } else {
    return (Idx)data_[element.element];
  }
}

template <typename T>
MeshDataMaterialSelector<T>::MeshDataMaterialSelector(const ID &name, SolidMechanicsModel &model,
                                                      Idx first_index)
    : ElementDataMaterialSelector<T>(model.getMesh().template getData<T>(name), model,
                                     first_index) {}

inline Array<Idx> Material::getElementFilter(ElementType) const {
  const auto &mat = model_->getElementMaterials();
  Int n = 0;
  for (Idx m : mat) n += m == index_;
  Array<Idx> out(n, 1);
  Int k = 0;
  for (size_t e = 0; e < mat.size(); ++e)
    if (mat[e] == index_) out(k++, 0) = (Idx)e;
  return out;
}

inline Real Material::get(const ID &param) const {
  Real v = 0;
  check(akb_model_get_material_param(model_->handle(), index_, param.c_str(), &v));
  return v;
}
inline ID Material::getName() const {
  char buf[256];
  check(akb_model_get_material_name(model_->handle(), index_, buf, sizeof(buf)));
  return buf;
}
inline Array<Real> Material::qp(int field) {
  model_->syncUp();
  int64_t n = 0;
  check(akb_model_qp_field_size(model_->handle(), field, index_, &n));
  const Int comps = (field == AKB_ISO_HARDENING || field == AKB_PLASTIC_ENERGY)
                        ? 1
                        : model_->getSpatialDimension() * model_->getSpatialDimension();
  Array<Real> out(n / comps, comps);
  check(akb_model_get_qp_field(model_->handle(), field, index_, out.data(), n));
  return out;
}
inline Array<Real> Material::getStress(ElementType) { return qp(AKB_STRESS); }
inline Array<Real> Material::getGradU(ElementType) { return qp(AKB_GRAD_U); }
inline int Material::internalId(const ID &name) {
  static const std::map<ID, int> ids = {
      {"stress", AKB_STRESS}, {"grad_u", AKB_GRAD_U},
      {"piola_kirchhoff_2", AKB_PIOLA_KIRCHHOFF_2}, {"inelastic_strain", AKB_INELASTIC_STRAIN},
      {"iso_hardening", AKB_ISO_HARDENING}, {"plastic_energy", AKB_PLASTIC_ENERGY},
      {"eigen_grad_u", AKB_EIGEN_GRAD_U}};
  return ids.at(name);
}
inline Array<Real> Material::getInternal(const ID &name, ElementType) {
  return qp(internalId(name));
}
inline void Material::setInternal(const ID &name, const Array<Real> &values, ElementType) {
  const int field = internalId(name);
  int64_t n = 0;
  check(akb_model_qp_field_size(model_->handle(), field, index_, &n));
  if ((int64_t)(values.size() * values.getNbComponent()) != n)
    throw Exception(AKB_EINVAL, "setInternal: size mismatch for " + name);
  check(akb_model_set_qp_field(model_->handle(), field, index_, values.data(), n));
}

/* ---- Server: many solves resident on one GPU ----------------------------- */
// RAII wrapper of akb_server_*: submit() copies the request's inputs, the
// result arrays passed in the request are filled before poll() reports it.
class Server {
public:
  explicit Server(const akb_server_config &cfg = akb_server_config{}) {
    check(akb_server_create(&cfg, &h_));
  }
  ~Server() {
    if (h_) akb_server_destroy(h_);
  }
  Server(const Server &) = delete;
  Server &operator=(const Server &) = delete;

  int64_t submit(const akb_request &request) {
    int64_t id = 0;
    check(akb_server_submit(h_, &request, &id));
    return id;
  }
  std::vector<akb_completion> poll(double wait_seconds = 0., int capacity = 64) {
    std::vector<akb_completion> out((size_t)capacity);
    int n = 0;
    check(akb_server_poll(h_, out.data(), capacity, &n, wait_seconds));
    out.resize((size_t)n);
    return out;
  }
  akb_server_stats stats() {
    akb_server_stats st{};
    check(akb_server_get_stats(h_, &st));
    return st;
  }

private:
  akb_server *h_ = nullptr;
};

}  // namespace akantu_b200

#endif
