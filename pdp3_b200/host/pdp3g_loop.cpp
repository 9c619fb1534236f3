// pdp3g_loop: the PDP3 main loop (LoadInitParam::run, src/loadInitParam.cpp:
// 455-589, and init_beam :168-248) written against the upstream-style classes
// of pdp3_classes.h, i.e. the call sequence a PDP3 host keeps when it links
// the B200 step instead of the CPU one.
//
//   pdp3g_loop <case_dir> <steps> <out_dir>
//
// <case_dir>/case.txt holds "key value" lines: r_size z_size n_grid_r n_grid_z
// dt current_time pml_l1 pml_l2 pml_l3 pml_sigma1 pml_sigma2 pusher precision
// n_species, per species s: species<s>_charge species<s>_mass species<s>_n,
// and optionally beam_charge beam_mass beam_number_macro beam_length
// beam_radius beam_density beam_velocity beam_number_bunches beam_distance.
// Species arrays are raw float64 files species<s>_{r,z,vr,vphi,vz,w}.f64, or,
// with keys species<s>_left_density species<s>_right_density
// species<s>_temperature, the upstream's own initial state (init_particles:
// load_cylindrical_spatial_distribution + velocity_distribution).
// Optional <case_dir>/names.txt: the species' names, one per line (default
// species<s>).  Optional <case_dir>/probes.txt: one ProbePlain per line,
//   <type> <component> <start_r> <start_z> <end_r> <end_z> <schedule> [<specie>]
// (type 0 frame, 1 col, 2 row, 3 dot, 4 mpframe; an mpframe's component
// names a species or Beam#<k>; components T and density take the species as
// <specie>),
// written under <out_dir>/probes
// by dump_data's schedule test after every step (key dump_frames_per_file,
// default 1).  The loop writes E_r.. J_z (raw float64
// [n_grid_r*n_grid_z]) and every species' r, z, vr, vphi, vz, alive to
// <out_dir>, and prints one JSON line.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "pdp3_classes.h"

using namespace pdp3gpu;

static std::map<std::string, double> read_case(const std::string &dir) {
  std::map<std::string, double> kv;
  std::ifstream f(dir + "/case.txt");
  std::string key;
  double v;
  while (f >> key >> v) kv[key] = v;
  return kv;
}

static std::vector<double> read_f64(const std::string &path, size_t n) {
  std::vector<double> a(n);
  FILE *fp = fopen(path.c_str(), "rb");
  if (!fp || fread(a.data(), sizeof(double), n, fp) != n) {
    fprintf(stderr, "cannot read %s\n", path.c_str());
    exit(2);
  }
  fclose(fp);
  return a;
}

static void write_raw(const std::string &path, const void *data, size_t bytes) {
  FILE *fp = fopen(path.c_str(), "wb");
  if (!fp) return;
  fwrite(data, 1, bytes, fp);
  fclose(fp);
}

int main(int argc, char **argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s <case_dir> <steps> <out_dir>\n", argv[0]);
    return 1;
  }
  const std::string cdir = argv[1], odir = argv[3];
  const int steps = atoi(argv[2]);
  auto kv = read_case(cdir);
  auto get = [&](const std::string &k, double def = 0.0) {
    auto it = kv.find(k);
    return it == kv.end() ? def : it->second;
  };
  try {
    // Parameters: geometry, PML, time (src/parameters.cpp:215-268)
    Geometry geom(get("r_size"), get("z_size"), (int)get("n_grid_r"), (int)get("n_grid_z"));
    geom.set_epsilon();
    if (get("pml_l1") != 0 || get("pml_l2") != 0 || get("pml_l3") != 0)
      geom.set_pml(get("pml_l1"), get("pml_l2"), get("pml_l3"), get("pml_sigma1"),
                   get("pml_sigma2"));
    Time time(get("current_time"), 0.0, 0.0, get("current_time") + steps * get("dt"), get("dt"));
    Device &dev = Device::of(&geom);
    dev.pusher = (int)get("pusher");
    dev.precision = (int)get("precision");
    // init_fields (src/loadInitParam.cpp:250-260)
    EField efield(&geom);
    HField hfield(&geom);
    efield.boundary_conditions();
    efield.set_homogeneous_efield(0., 0., 0.);
    hfield.set_homogeneous_h(0., 0., 0.);
    efield.set_fi_on_z();
    // init_particles (src/loadInitParam.cpp:134-166), state given explicitly
    ParticlesList p_list;
    ChargeDensity c_rho_new(&geom), c_rho_old(&geom), c_rho_bunch(&geom);
    Current c_current(&geom);
    std::vector<std::unique_ptr<Particles>> owned;
    const int nsp = (int)get("n_species");
    std::vector<std::string> species_names;
    {
      std::ifstream nf(cdir + "/names.txt");
      std::string nm;
      while ((int)species_names.size() < nsp && nf >> nm) species_names.push_back(nm);
      for (int s = (int)species_names.size(); s < nsp; s++)
        species_names.push_back("species" + std::to_string(s));
    }
    for (int s = 0; s < nsp; s++) {
      const std::string p = "species" + std::to_string(s) + "_";
      const size_t n = (size_t)get(p + "n");
      if (kv.count(p + "temperature")) {
        // LoadInitParam::init_particles (src/loadInitParam.cpp:157-164)
        owned.emplace_back(new Particles(species_names[s].c_str(), get(p + "charge"),
                                         get(p + "mass"), (int)n, &geom));
        Particles *prt = owned.back().get();
        prt->load_cylindrical_spatial_distribution(get(p + "left_density"),
                                                   get(p + "right_density"), 0);
        prt->velocity_distribution(get(p + "temperature"));
        p_list.part_list.push_back(prt);
        continue;
      }
      auto r = read_f64(cdir + "/" + p + "r.f64", n), z = read_f64(cdir + "/" + p + "z.f64", n);
      auto vr = read_f64(cdir + "/" + p + "vr.f64", n);
      auto vp = read_f64(cdir + "/" + p + "vphi.f64", n);
      auto vz = read_f64(cdir + "/" + p + "vz.f64", n), w = read_f64(cdir + "/" + p + "w.f64", n);
      owned.emplace_back(new Particles(species_names[s].c_str(), get(p + "charge"), get(p + "mass"),
                                       (int)n, &geom));
      Particles *prt = owned.back().get();
      for (size_t i = 0; i < n; i++) {
        prt->pos[i][0] = r[i];
        prt->pos[i][1] = 0.0;
        prt->pos[i][2] = z[i];
        prt->vel[i][0] = vr[i];
        prt->vel[i][1] = vp[i];
        prt->vel[i][2] = vz[i];
        prt->charge_array[i] = prt->charge * w[i];
        prt->mass_array[i] = prt->mass * w[i];
      }
      p_list.part_list.push_back(prt);
    }
    // init_beam state (src/loadInitParam.cpp:168-248)
    const bool beam = get("beam_number_bunches") > 0;
    std::vector<Bunch *> c_bunches;
    int current_bunch_number = 0;
    auto init_beam = [&]() {
      if (!beam) return;
      const double duration = get("beam_length") / get("beam_velocity");
      const double hole_duration = get("beam_distance") / get("beam_velocity");
      const double bunch_inject_time = current_bunch_number * (duration + hole_duration);
      if (time.current_time >= bunch_inject_time &&
          current_bunch_number < (int)get("beam_number_bunches")) {
        char name[64];
        snprintf(name, sizeof(name), "Beam#%d", current_bunch_number);
        owned.emplace_back(new Bunch(name, get("beam_charge"), get("beam_mass"),
                                     (int)get("beam_number_macro"), &geom, duration,
                                     get("beam_radius"), get("beam_density"),
                                     get("beam_velocity"), current_bunch_number, hole_duration));
        Bunch *b = static_cast<Bunch *>(owned.back().get());
        p_list.part_list.push_back(b);
        species_names.push_back(name);
        c_bunches.push_back(b);
        ++current_bunch_number;
      }
      for (Bunch *b : c_bunches) b->bunch_inject(&time);
    };
    // probes (LoadInitParam::init_probes / dump_data)
    std::vector<std::unique_ptr<ProbePlain>> probe_store;
    std::vector<ProbePlain *> probes;
    {
      std::ifstream pf(cdir + "/probes.txt");
      std::string line;
      while (std::getline(pf, line)) {
        std::istringstream ls(line);
        int type, r0, z0, r1, z1, sched;
        std::string comp, specie = "none";
        if (!(ls >> type >> comp >> r0 >> z0 >> r1 >> z1 >> sched)) continue;
        ls >> specie;
        probe_store.emplace_back(new ProbePlain((odir + "/probes").c_str(), comp.c_str(), type, r0,
                                                z0, r1, z1, false, 0, sched, specie.c_str()));
        probes.push_back(probe_store.back().get());
      }
    }
    const int frames_per_file = (int)get("dump_frames_per_file", 1);
    // LoadInitParam::run (src/loadInitParam.cpp:471-587)
    auto t0 = std::chrono::steady_clock::now();
    int done = 0;
    while (done < steps) {
      init_beam();
      hfield.calc_field(&efield, &time);
      c_current.reset_j();
      c_rho_old.reset_rho();
      c_rho_bunch.reset_rho();
      p_list.step_v(&efield, &hfield, &time);
      p_list.full_current_distribution(&c_current, &time);
      efield.calc_field(&hfield, &time, &c_current);
      c_rho_new.reset_rho();
      if (!probes.empty())
        dump_probes(probes, Device::of(&geom).ctx(&time), &time, frames_per_file, species_names);
      time.current_time = time.current_time + time.delta_t;
      ++done;
    }
    auto t1 = std::chrono::steady_clock::now();
    // outputs
    efield.download();
    hfield.download();
    const size_t ng = (size_t)geom.n_grid_r * geom.n_grid_z;
    write_raw(odir + "/E_r.f64", efield.field_r[0], ng * 8);
    write_raw(odir + "/E_phi.f64", efield.field_phi[0], ng * 8);
    write_raw(odir + "/E_z.f64", efield.field_z[0], ng * 8);
    write_raw(odir + "/H_r.f64", hfield.field_r[0], ng * 8);
    write_raw(odir + "/H_phi.f64", hfield.field_phi[0], ng * 8);
    write_raw(odir + "/H_z.f64", hfield.field_z[0], ng * 8);
    write_raw(odir + "/J_r.f64", c_current.get_j_r()[0], ng * 8);
    write_raw(odir + "/J_phi.f64", c_current.get_j_phi()[0], ng * 8);
    write_raw(odir + "/J_z.f64", c_current.get_j_z()[0], ng * 8);
    for (size_t s = 0; s < p_list.part_list.size(); s++) {
      Particles *p = p_list.part_list[s];
      p->download();
      std::vector<double> a(p->number);
      std::vector<uint8_t> alive(p->number);
      const char *names[5] = {"r", "z", "vr", "vphi", "vz"};
      for (int c = 0; c < 5; c++) {
        for (unsigned i = 0; i < p->number; i++)
          a[i] = c == 0 ? p->pos[i][0] : c == 1 ? p->pos[i][2] : p->vel[i][c - 2];
        write_raw(odir + "/out" + std::to_string(s) + "_" + names[c] + ".f64", a.data(),
                  a.size() * 8);
      }
      for (unsigned i = 0; i < p->number; i++) alive[i] = p->is_alive[i] ? 1 : 0;
      write_raw(odir + "/out" + std::to_string(s) + "_alive.u8", alive.data(), alive.size());
    }
    printf("{\"steps\": %d, \"seconds\": %.6f, \"species\": %zu, \"time\": %.17g}\n", done,
           std::chrono::duration<double>(t1 - t0).count(), p_list.part_list.size(),
           time.current_time);
  } catch (const Error &e) {
    fprintf(stderr, "pdp3g_loop: %s\n", e.what());
    return 3;
  }
  return 0;
}
