// host_mirror.cpp -- drives the C++ host mirror (include/salmon_b200.hpp) the
// way SALMON's Fortran drives hpsi / taylor, for the parity tests.
//
// usage: host_mirror <input> <output>
// Both files are sequences of records
//   uint32 name length, name, uint32 kind (0 int32, 1 float64), uint64 count, data
// The input holds the reference-layout arrays of one system (written by
// tests/test_cpp_host.py); the output holds H psi, T psi, the Taylor step,
// calc_eigen_energy, calc_current, calc_density and the status code that an
// invalid (aliased) hpsi call raises.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "salmon_b200.hpp"

namespace {

struct Record {
  uint32_t kind = 0;
  std::vector<char> bytes;
};

std::map<std::string, Record> read_records(const char* path) {
  std::map<std::string, Record> m;
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error(std::string("cannot open ") + path);
  for (;;) {
    uint32_t nlen = 0;
    if (!f.read(reinterpret_cast<char*>(&nlen), 4)) break;
    std::string name(nlen, '\0');
    f.read(&name[0], nlen);
    Record r;
    uint64_t count = 0;
    f.read(reinterpret_cast<char*>(&r.kind), 4);
    f.read(reinterpret_cast<char*>(&count), 8);
    r.bytes.resize(count * (r.kind == 0 ? 4 : 8));
    f.read(r.bytes.data(), (std::streamsize)r.bytes.size());
    if (!f) throw std::runtime_error("truncated record " + name);
    m[name] = std::move(r);
  }
  return m;
}

template <typename T>
std::vector<T> get(const std::map<std::string, Record>& m, const std::string& name) {
  auto it = m.find(name);
  if (it == m.end()) throw std::runtime_error("missing record " + name);
  std::vector<T> v(it->second.bytes.size() / sizeof(T));
  if (!v.empty()) std::memcpy(v.data(), it->second.bytes.data(), it->second.bytes.size());
  return v;
}

void put(std::ofstream& f, const std::string& name, const double* p, size_t n) {
  const uint32_t nlen = (uint32_t)name.size(), kind = 1;
  const uint64_t count = n;
  f.write(reinterpret_cast<const char*>(&nlen), 4);
  f.write(name.data(), nlen);
  f.write(reinterpret_cast<const char*>(&kind), 4);
  f.write(reinterpret_cast<const char*>(&count), 8);
  f.write(reinterpret_cast<const char*>(p), (std::streamsize)(n * sizeof(double)));
}

template <size_t N>
void fill(int (&dst)[N], const std::vector<int>& src) {
  for (size_t i = 0; i < N; ++i) dst[i] = src.at(i);
}

}  // namespace

int main(int argc, char** argv) {
  namespace sb = salmon_b200;
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s <input> <output>\n", argv[0]);
    return 2;
  }
  try {
    const auto in = read_records(argv[1]);
    sb::s_rgrid mg;
    fill(mg.is, get<int>(in, "is"));
    fill(mg.ie, get<int>(in, "ie"));
    fill(mg.is_array, get<int>(in, "is_array"));
    fill(mg.ie_array, get<int>(in, "ie_array"));
    fill(mg.lg_num, get<int>(in, "lg_num"));
    mg.idx = get<int>(in, "idx");
    mg.idy = get<int>(in, "idy");
    mg.idz = get<int>(in, "idz");
    sb::s_stencil st;
    st.coef_lap0 = get<double>(in, "coef_lap0").at(0);
    const auto lap = get<double>(in, "coef_lap"), nab = get<double>(in, "coef_nab");
    for (int i = 0; i < 12; ++i) {
      st.coef_lap[i] = lap.at(i);
      st.coef_nab[i] = nab.at(i);
    }
    sb::s_dft_system sys;
    const auto dims = get<int>(in, "nspin_no_nk");
    sys.nspin = dims.at(0);
    sys.no = dims.at(1);
    sys.nk = dims.at(2);
    const auto hgs = get<double>(in, "hgs");
    for (int d = 0; d < 3; ++d) sys.hgs[d] = hgs.at(d);
    sys.hvol = get<double>(in, "hvol").at(0);
    sys.vec_k = get<double>(in, "vec_k");
    sys.rocc = get<double>(in, "rocc");
    sys.wtk = get<double>(in, "wtk");
    const auto ac = get<double>(in, "vec_Ac");
    for (int d = 0; d < 3; ++d) sys.vec_Ac[d] = ac.at(d);
    const auto V = get<double>(in, "V_local");
    const size_t nint = V.size() / sys.nspin;
    std::vector<sb::s_scalar> V_local(sys.nspin);
    for (int s = 0; s < sys.nspin; ++s) V_local[s].f.assign(V.begin() + s * nint, V.begin() + (s + 1) * nint);
    sb::s_pp_grid pp;
    const auto ppd = get<int>(in, "natom_nps_nlma");
    pp.natom = ppd.at(0);
    pp.nps = ppd.at(1);
    pp.nlma = ppd.at(2);
    pp.mps = get<int>(in, "mps");
    pp.jxyz = get<int>(in, "jxyz");
    pp.rxyz = get<double>(in, "rxyz");
    pp.uv = get<double>(in, "uv");
    pp.ia_tbl = get<int>(in, "ia_tbl");
    pp.rinv_uvu = get<double>(in, "rinv_uvu");
    sb::s_rt rt;
    const auto zc = get<double>(in, "zc");
    for (size_t i = 0; i + 1 < zc.size(); i += 2) rt.zc.emplace_back(zc[i], zc[i + 1]);
    const auto zwf_d = get<double>(in, "zwf");
    std::vector<std::complex<double>> zwf(zwf_d.size() / 2);
    std::memcpy(zwf.data(), zwf_d.data(), zwf_d.size() * sizeof(double));

    sb::context ctx(0, mg, st, sys, V_local, pp);
    sb::s_orbital tpsi(ctx), htpsi(ctx), ttpsi(ctx), out(ctx), work(ctx);
    tpsi.from_ref(zwf.data());
    std::vector<std::complex<double>> buf(zwf.size());
    std::ofstream of(argv[2], std::ios::binary);

    sb::hpsi(ctx, tpsi, htpsi, ttpsi, sys);
    htpsi.to_ref(buf.data());
    put(of, "htpsi", reinterpret_cast<const double*>(buf.data()), 2 * buf.size());
    ttpsi.to_ref(buf.data());
    put(of, "ttpsi", reinterpret_cast<const double*>(buf.data()), 2 * buf.size());

    std::vector<double> esp;
    double ekin = 0.0, enl = 0.0;
    sb::calc_eigen_energy(ctx, tpsi, htpsi, ttpsi, sys, esp, ekin, enl);
    put(of, "esp", esp.data(), esp.size());
    put(of, "ekin", &ekin, 1);
    put(of, "enl", &enl, 1);

    std::vector<double> curr(3 * sys.nspin);
    sb::calc_current(ctx, tpsi, sys.vec_Ac, curr.data());
    put(of, "curr", curr.data(), curr.size());
    std::vector<sb::s_scalar> rho(sys.nspin);
    for (auto& r : rho) r.f.assign(nint, 0.0);
    sb::calc_density(ctx, rho, tpsi);
    for (int s = 0; s < sys.nspin; ++s) put(of, "rho" + std::to_string(s), rho[s].f.data(), nint);


    sb::taylor(ctx, sys, tpsi, out, work, rt);  // tpsi is scratch afterwards
    out.to_ref(buf.data());
    put(of, "taylor", reinterpret_cast<const double*>(buf.data()), 2 * buf.size());

    // the reference stops on an invalid call; the mirror throws with the code
    double code = 0.0;
    try {
      sb::hpsi(ctx, out, out, sys);
    } catch (const sb::error& e) {
      code = e.code();
    }
    put(of, "alias_code", &code, 1);

    // the self-consistent potential of this density (periodic, nspin = 1)
    const auto brl = get<double>(in, "primitive_b");
    sb::s_scalar vh, vpsl;
    std::vector<sb::s_scalar> vxc;
    double exc = 0.0;
    sb::hartree(ctx, brl.data(), rho[0], vh);
    sb::exchange_correlation(ctx, rho[0], vxc, exc);
    put(of, "Vh", vh.f.data(), nint);
    put(of, "Vxc", vxc[0].f.data(), nint);
    put(of, "E_xc", &exc, 1);
    vpsl.f = V_local[0].f;
    sb::update_vlocal(ctx, vh, vpsl, vxc);
    tpsi.from_ref(zwf.data());  // tpsi was the Taylor step's scratch
    sb::hpsi(ctx, tpsi, htpsi, sys);
    htpsi.to_ref(buf.data());
    put(of, "htpsi_scf", reinterpret_cast<const double*>(buf.data()), 2 * buf.size());
    ctx.sync();
  } catch (const std::exception& e) {
    std::fprintf(stderr, "host_mirror: %s\n", e.what());
    return 1;
  }
  return 0;
}
