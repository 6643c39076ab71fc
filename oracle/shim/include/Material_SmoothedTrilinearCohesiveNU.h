/* Declaration of TrilinearSmoothedCohesiveNUMaterial for the oracle build of the reference (test
 * infrastructure only).  The reference ships src/Material_SmoothedTrilinearCohesiveNU.cpp without
 * this header; the class is declared here from the members that .cpp defines and uses: the four
 * curve parameters and the fracture energy with their "set" flags, the mode-mixity and contact
 * parameters, and the parameter setters that derive a missing parameter from the others. */
#pragma once
#include "material.h"

class TrilinearSmoothedCohesiveNUMaterial : public Material {
 protected:
  double _sigma_c, _delta_c1, _delta_c2, _delta_c3, _G, _beta2, _alpha;
  bool _s_set, _d1_set, _d2_set, _d3_set, _G_set;
  bool ready;
  void set_sc(double sc);
  double get_sc();
  void set_dc1(double dc);
  double get_dc1();
  void set_dc2(double dc);
  double get_dc2();
  void set_dc3(double dc);
  double get_dc3();
  void set_G(double G);
  double get_G();
  void set_b(double b);
  void set_alpha(double a);
  double getDeltaEff(std::vector<double>& delta_ttn);

 public:
  TrilinearSmoothedCohesiveNUMaterial();
  virtual ~TrilinearSmoothedCohesiveNUMaterial() {}
  virtual Material::output_params* Constitutive(Material::input_params& input);
  virtual material_type get_type() { return TL_COHESIVE_NO_UNLOADING; }
  virtual classification get_classification() { return STRUCTURAL; }
  virtual bool linear() { return false; }
  virtual void set_parameter(std::string name, double val);
  virtual double get_parameter(std::string name);
  virtual bool is_cohesive() { return true; }
  virtual id_type get_cohesive_damage_zone(std::vector<double>& delta);
  virtual double getNormalizedCohesiveFailure(std::vector<double>& delta_ntt);
  virtual Material* allocate();
  virtual void copy(Material* other_mat);
  virtual SensitivityMaterialParameter* getSensitivityParameter(std::string name);
  virtual Material::sensitivity_output_params* SensitivityConstitutive(Material::sensitivity_input_params& input);
};
