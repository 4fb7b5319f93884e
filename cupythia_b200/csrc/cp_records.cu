// cp_records.cu -- host-side consumers of the 64-byte event records: colour tags of the encoded
// colour flow, and a Les Houches Event File (LHEF 3.0) writer.  Host code only: these entry
// points need no GPU.
//
// The LHEF layout follows the Les Houches accord as the reference writes it
// (cuPythia/pipeline/lhe_writer.cu:46-70, cuPythia/07_unweighting_lhe/unweight_lhe.cu:74-102):
// <init> with the beam line (IDBMUP EBMUP PDFGUP PDFSUP IDWTUP NPRUP) and one line per process
// (XSECUP XERRUP XMAXUP LPRUP), then one <event> per record with NUP IDPRUP XWGTUP SCALUP AQEDUP
// AQCDUP and one line per parton (IDUP ISTUP MOTHUP1 MOTHUP2 ICOLUP1 ICOLUP2 PUP1..5 VTIMUP
// SPINUP).  Unlike the reference (one process, a fixed gg -> gg colour ring) every record
// carries its own process code and the colour flow its setIdColAcol chose.
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>
#if defined(__linux__)
#include <sched.h>
#endif
#include "cp_internal.cuh"

extern "C" int cp_colour_tags(uint16_t process, uint16_t colour, int col[4], int acol[4])
{
  if (!col || !acol) return CP_ERR_INVALID;
  return cp_colour_expand(process, colour, col, acol) ? CP_OK : CP_ERR_INVALID;
}

// One event's Sigma2*::setIdColAcol on the host, with the record builder's code (cp_colour_flow,
// cp_colour_expand) at FP32: the outgoing flavours and the colour tags of process `code` for the
// incoming pair (id1, id2) at tHat/sHat = t_over_s, uHat/sHat = u_over_s.
extern "C" int cp_set_id_col_acol(int code, int id1, int id2, double t_over_s, double u_over_s, int n_quark_new,
                                  double r_flavour, double r_colour, double r_swap, int ids_out[4], int col[4],
                                  int acol[4])
{
  if (code < 111 || code > 115 || !ids_out || !col || !acol || !(t_over_s < 0.0) || !(u_over_s < 0.0) ||
      n_quark_new < 1 || n_quark_new > 5)
    return CP_ERR_INVALID;
  const bool gin1 = id1 == 21, gin2 = id2 == 21;
  const bool q1 = id1 != 0 && id1 >= -5 && id1 <= 5, q2 = id2 != 0 && id2 >= -5 && id2 <= 5;
  const bool ok = (code == 111 || code == 112) ? (gin1 && gin2)
                  : code == 113                ? ((q1 && gin2) || (gin1 && q2))
                  : code == 114                ? (q1 && q2)
                                               : (q1 && q2 && id2 == -id1);
  if (!ok) return CP_ERR_INVALID;
  int id[4] = {id1, id2, id1, id2};
  if (code == 111 || code == 115) { id[2] = 21; id[3] = 21; }
  if (code == 112) {
    int qn = 1 + (int)((float)n_quark_new * (float)r_flavour);
    if (qn > n_quark_new) qn = n_quark_new;
    id[2] = qn;
    id[3] = -qn;
  }
  const uint32_t flow = cp_colour_flow(code, id, (float)t_over_s, (float)u_over_s, (float)r_colour, (float)r_swap);
  if (!cp_colour_expand((uint16_t)code, (uint16_t)flow, col, acol)) return CP_ERR_INVALID;
  for (int k = 0; k < 4; ++k) ids_out[k] = id[k];
  return CP_OK;
}

// LHEF tag of a colour index (0 = none)
static inline int lhef_tag(int c) { return c ? 500 + c : 0; }

// The <event> blocks of events [a, b) appended to out; false if a record's process code or
// colour flow is invalid.
static bool lhef_events(const cp_config* cfg, const CpHadParams& P, const cp_event* events, uint64_t a, uint64_t b,
                        std::string& out)
{
  char line[512];
  out.clear();
  out.reserve((size_t)(b - a) * 560);
  auto put = [&](int len) {
    if (len > 0) out.append(line, (size_t)(len < (int)sizeof line ? len : (int)sizeof line - 1));
  };
  for (uint64_t i = a; i < b; ++i) {
    const cp_event& e = events[i];
    int col[4], acol[4];
    if (cp_colour_tags(e.process, e.colour, col, acol) != CP_OK) return false;
    const double pT2 = (double)e.pt_hat * e.pt_hat;
    const double scale = sqrt(pT2 * cfg->k_fac);
    const double aS = cp_alphas(P, (float)(pT2 * cfg->k_ren));
    out.append("<event>\n");
    // NUP IDPRUP XWGTUP SCALUP AQEDUP AQCDUP
    put(snprintf(line, sizeof line, "4 %d %.8E %.8E 7.8175100E-03 %.8E\n", (int)e.process, (double)e.weight, scale, aS));
    // IDUP ISTUP MOTHUP1 MOTHUP2 ICOLUP1 ICOLUP2 PX PY PZ E M VTIMUP SPINUP
    for (int k = 0; k < 2; ++k)
      put(snprintf(line, sizeof line,
                   "%d -1 0 0 %d %d 0.0000000000E+00 0.0000000000E+00 %.10E %.10E 0.0000000000E+00 0. 9.\n",
                   (int)e.id[k], lhef_tag(col[k]), lhef_tag(acol[k]), (double)e.pz_in[k], fabs((double)e.pz_in[k])));
    const float* p[2] = {e.p3, e.p4};
    for (int k = 0; k < 2; ++k)
      put(snprintf(line, sizeof line, "%d 1 1 2 %d %d %.10E %.10E %.10E %.10E 0.0000000000E+00 0. 9.\n",
                   (int)e.id[2 + k], lhef_tag(col[2 + k]), lhef_tag(acol[2 + k]), (double)p[k][0], (double)p[k][1],
                   (double)p[k][2], (double)p[k][3]));
    out.append("</event>\n");
  }
  return true;
}

// host threads this process may run on (its CPU affinity), at most 64
static int lhef_threads()
{
#if defined(__linux__)
  cpu_set_t set;
  CPU_ZERO(&set);
  if (sched_getaffinity(0, sizeof set, &set) == 0) {
    const int c = CPU_COUNT(&set);
    if (c > 0) return c < 64 ? c : 64;
  }
#endif
  const unsigned c = std::thread::hardware_concurrency();
  return c ? (c < 64 ? (int)c : 64) : 1;
}

extern "C" int cp_write_lhef(const cp_config* cfg, const cp_event* events, uint64_t n, double sigma_mb,
                             double sigma_err_mb, const char* path)
{
  if (!cfg || (n && !events) || !path) return CP_ERR_INVALID;
  CpHadParams P{};
  const CpHadConfig hc{cfg->sqrt_s, cfg->pt_hat_min, cfg->alphas_mz, cfg->k_ren, cfg->k_fac, cfg->convert2mb,
                       cfg->n_quark_in, cfg->n_quark_new, cfg->proc_mask};
  if (cp_build_had_params(hc, P)) return CP_ERR_INVALID;
  FILE* f = fopen(path, "w");
  if (!f) return CP_ERR_INVALID;
  const double eBeam = 0.5 * cfg->sqrt_s;
  const double mb2pb = 1e9;
  // per-process counts and summed weights: XSECUP_k = sigma * (sum of weights of k) / (sum of weights)
  double wsum[5] = {0, 0, 0, 0, 0}, wtot = 0.0, wmax = 0.0;
  for (uint64_t i = 0; i < n; ++i) {
    const int code = events[i].process;
    if (code < 111 || code > 115) { fclose(f); return CP_ERR_INVALID; }
    wsum[code - 111] += events[i].weight;
    wtot += events[i].weight;
    wmax = events[i].weight > wmax ? events[i].weight : wmax;
  }
  int nproc = 0;
  for (int k = 0; k < 5; ++k) nproc += wsum[k] > 0 ? 1 : 0;
  fprintf(f, "<LesHouchesEvents version=\"3.0\">\n<header>\n");
  fprintf(f, "  cupythia_b200 unweighted pp -> 2 jets, sqrt(s) = %.1f GeV, pT_hat > %.2f GeV, CTEQ5L,\n",
          cfg->sqrt_s, cfg->pt_hat_min);
  fprintf(f, "  alpha_s(mZ) = %.4f first order, mu_R^2 = %.3g pT^2, mu_F^2 = %.3g pT^2; %llu events\n",
          cfg->alphas_mz, cfg->k_ren, cfg->k_fac, (unsigned long long)n);
  fprintf(f, "</header>\n<init>\n");
  // IDBMUP1 IDBMUP2 EBMUP1 EBMUP2 PDFGUP1 PDFGUP2 PDFSUP1 PDFSUP2 IDWTUP NPRUP
  // (PDFSUP 19051 = CTEQ5L in the LHAPDF numbering; IDWTUP 3: unit-weight events)
  fprintf(f, "2212 2212 %.10E %.10E 0 0 19051 19051 3 %d\n", eBeam, eBeam, nproc);
  for (int k = 0; k < 5; ++k) {
    if (wsum[k] <= 0) continue;
    const double frac = wsum[k] / wtot;
    const double xs = sigma_mb * mb2pb * frac;
    const double xe = mb2pb * sqrt(sigma_err_mb * sigma_err_mb * frac * frac +
                                   sigma_mb * sigma_mb * frac * (1.0 - frac) / (n > 0 ? (double)n : 1.0));
    fprintf(f, "%.10E %.10E %.10E %d\n", xs, xe, wmax, 111 + k);
  }
  fprintf(f, "</init>\n");
  // the <event> blocks: host threads format chunks of 8192 events each into their own buffer,
  // the calling thread writes the buffers in event order (the same bytes as one thread writing)
  const uint64_t chunk = 8192;
  const int nt = n > chunk ? lhef_threads() : 1;
  std::vector<std::string> bufs((size_t)nt);
  for (uint64_t base = 0; base < n; base += chunk * (uint64_t)nt) {
    std::atomic<int> bad{0};
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) {
      const uint64_t a = base + (uint64_t)t * chunk;
      if (a >= n) break;
      const uint64_t b = a + chunk < n ? a + chunk : n;
      th.emplace_back([&, t, a, b] {
        if (!lhef_events(cfg, P, events, a, b, bufs[(size_t)t])) bad = 1;
      });
    }
    if (!lhef_events(cfg, P, events, base, base + chunk < n ? base + chunk : n, bufs[0])) bad = 1;
    for (std::thread& x : th) x.join();
    if (bad) { fclose(f); return CP_ERR_INVALID; }
    for (int t = 0; t <= (int)th.size(); ++t) fwrite(bufs[(size_t)t].data(), 1, bufs[(size_t)t].size(), f);
  }
  fprintf(f, "</LesHouchesEvents>\n");
  const int bad = ferror(f);
  fclose(f);
  return bad ? CP_ERR_INVALID : CP_OK;
}
