/*
 * rk4_gpu.c - GPU drivers for NcorpiON's brute-force and mesh integrations.
 *
 * Drop-in replacements of integration_brute_force_SABA1 (src/rk4.c:840-954)
 * and integration_mesh (src/rk4.c:662-837).  They are compiled against the
 * reference's own headers (parameters.h, structure.h, rk4.h, display.h ...)
 * and linked with its objects and libncgpu.so; main.c reaches them through
 *     -Dintegration_brute_force_SABA1=ncgpu_integration_brute_force_SABA1
 *     -Dintegration_mesh=ncgpu_integration_mesh
 * on main.c's compile line only (the reference's rk4.o keeps its own copies).
 *
 * Bodies live on the GPU between calls.  The host keeps what the reference
 * keeps on the host: initial conditions (populate), the output files (readme,
 * resume, the first and last display), the progress printout, the mesh size
 * gamma (updated with the host's libm pow) and the brute-force switch.  At an
 * output step the half backward drift or kick of the printed copy runs on a
 * device snapshot and the cartesian files' text is formatted on the device
 * (gpu_display_device); stat.txt's line is printed here.  A step whose
 * progress is printed prints end_of_timestep's lines from the device's
 * statistics (gpu_progress_printout); the state comes back to the host only
 * for the last output and where the host's own code needs it.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "parameters.h"
#include "structure.h"
#include "physics.h"
#include "collision.h"
#include "rk4.h"
#include "display.h"
#include "ncgpu.h"

static void gpu_check(int status, const char *what)
{
      if (status != NCGPU_OK) {
            fprintf(stderr, "Error : %s failed on the GPU: %s", what, ncgpu_strerror(status));
            if (status == NCGPU_E_CUDA) fprintf(stderr, " (%s)", ncgpu_last_error());
            fprintf(stderr, "\n");
            abort();
      }
}

/* struct ncgpu_params from the parameters.h macros */
static void gpu_params(struct ncgpu_params *p)
{
      ncgpu_default_params(p);
      p->par_G = G;
      p->par_softening_parameter = softening_parameter;
      p->par_central_mass_bool = central_mass_bool;
      p->par_mutual_bool = mutual_bool;
      p->par_collision_bool = collision_bool;
      p->par_brute_force_bool = brute_force_bool;
      p->par_mesh_bool = mesh_bool;
      p->par_collision_type = elastic_collision_bool ? NCGPU_COLLISION_ELASTIC
                        : inelastic_collision_bool ? NCGPU_COLLISION_INELASTIC
                        : instant_merger_bool ? NCGPU_COLLISION_MERGER : NCGPU_COLLISION_FRAGMENTATION;
      p->par_collision_parameter = collision_parameter;
      p->par_one_collision_only_bool = one_collision_only_bool;
#if mesh_bool
      p->par_collision_cube_cells = collision_cube_cells;
      p->par_how_many_neighbours = how_many_neighbours;
      p->par_collision_cube_min = collision_cube_min;
#endif
      p->par_switch_to_brute_force = switch_to_brute_force;
      p->par_gravity_mode = NCGPU_GRAVITY_EXACT;
      p->par_disruption_threshold = disruption_threshold;
      p->par_high_dumping_threshold = high_dumping_threshold;
      p->par_reduce_to_COM_bool = reduce_to_COM_bool;
      {
            int pq[4] = pq_min_max;
            p->par_N_tilde = N_tilde;
            for (int j = 0; j < 4; j++) p->par_pq_min_max[j] = pq[j];
      }
      p->par_mu_parameter = mu_parameter;
      p->par_nu_parameter = nu_parameter;
      p->par_C1_parameter = C1_parameter;
      p->par_k_parameter = k_parameter;
      p->par_merging_threshold = merging_threshold;
      p->par_fragment_threshold = fragment_threshold;
      p->par_J2_bool = J2_bool;
      p->par_J2 = J2_value;
      p->par_R_unit = R_unit;
      p->par_sideral_omega = SideralOmega;
      p->par_central_tides_bool = central_tides_bool;
      p->par_k2 = k2;
      p->par_Delta_t = Delta_t;
      p->par_dimensionless_moi = dimensionless_moi;
}

/* The GPU path covers the configurations of its hot path only. */
static void gpu_supported(void)
{
      if (inner_fluid_disk_bool || viscoelastic_bool || pert_mass > 0. || openGL_bool) {
            fprintf(stderr, "Error : the GPU integration does not cover the inner fluid disk, the viscoelastic "
                            "body, the perturber or the 3D viewer.\n");
            abort();
      }
}

static void gpu_upload(struct moonlet *moonlets)
{
      gpu_check(ncgpu_upload((const struct ncgpu_body *)moonlets, exists, largest_id, (const struct ncgpu_body *)&CM),
                "upload");
}

/* device state -> host arrays and the reference's globals */
static void gpu_pull(struct moonlet *moonlets)
{
      int lid;
      gpu_check(ncgpu_download((struct ncgpu_body *)moonlets, exists, &lid, (struct ncgpu_body *)&CM), "download");
      for (int j = lid + 1; j <= largest_id && j < N_max; j++) exists[j] = 0;
      largest_id = lid;
      /* the central body's rotation, which the device's tides change, and the
         host's J2 for its own kicks: the fluid-body J2 of the state at the
         last end of step (src/rk4.c:459-463); neither the rotation nor the
         central mass has changed since */
      if (central_tides_bool) gpu_check(ncgpu_get_sideral_omega(&SideralOmega), "sideral rotation");
      if (J2_bool && J2_value == 0.) J2 = 0.5 * SideralOmega * SideralOmega * R_unit * R_unit * R_unit / (G * CM.mass);
}

/* the output step's copy (device snapshot) -> buffer, the shared globals and
   CM_buffer, for an output the host prints itself */
static void gpu_snapshot_pull(struct moonlet *buffer)
{
      int lid;
      gpu_check(ncgpu_download((struct ncgpu_body *)buffer, exists, &lid, (struct ncgpu_body *)&CM_buffer), "download");
      for (int j = lid + 1; j <= largest_id && j < N_max; j++) exists[j] = 0;
      largest_id = lid;
      if (central_tides_bool) gpu_check(ncgpu_get_sideral_omega(&SideralOmega), "sideral rotation");
}

/* The collision records of the last sweep appended to collisionDatas, as
   collision() and merger() fill them (src/physics.c:608-622, 685-704). */
static void gpu_collision_records(double t_now)
{
      int n = 0;
      gpu_check(ncgpu_get_events(NULL, NULL, 0, &n), "events");
      if (n == 0) return;
      struct ncgpu_event *ev = (struct ncgpu_event *)malloc(sizeof(struct ncgpu_event) * (size_t)n);
      double *rec = (double *)malloc(sizeof(double) * 8 * (size_t)n);
      gpu_check(ncgpu_get_events(ev, rec, n, &n), "events");
#if write_collisions_bool
      if (write_to_files_bool) {
            for (int e = 0; e < n; e++) {
                  const double *r = rec + 8 * e;
                  double t = r[0], mA = r[1], mB = r[2], RA = r[3], RB = r[4], dV = r[5], drdv = r[6];
                  (collisionDatas + indexCollision)->time = t_now + t;
                  (collisionDatas + indexCollision)->m1 = mB;
                  (collisionDatas + indexCollision)->m2 = mA;
                  (collisionDatas + indexCollision)->R1 = RB;
                  (collisionDatas + indexCollision)->R2 = RA;
                  (collisionDatas + indexCollision)->DeltaV = dV;
                  (collisionDatas + indexCollision)->impact_angle = acos(-drdv / ((RA + RB) * dV));
                  (collisionDatas + indexCollision)->m_tilde = ev[e].type == NCGPU_COLLISION_MERGER         ? mA + mB
                                                               : ev[e].type == NCGPU_COLLISION_FRAGMENTATION ? r[7]
                                                                                                             : mA;
                  indexCollision++;
                  if (indexCollision == 2 * output_step * N_max) {
                        fprintf(stderr, "Error: The array collisionDatas is not large enough.\n");
                        abort();
                  }
            }
      }
#endif
      free(ev);
      free(rec);
}

/* display() (src/display.c:239-451) of the device state -- the output step's
   copy.  The cartesian files' text comes formatted from the device
   (ncgpu_format_cartesian).  The elliptic files' elements come from the
   device's cart2ell (ncgpu_elliptic_begin): the mean longitude's atan2 is this
   C library's (ncgpu_host_atan2), and the bodies the device lists (hyperbolic
   orbits, the (k, h) warning, NaNs) go through the reference's own cart2ell,
   which prints its warnings in slot order as display()'s loop does; the device
   then formats the six files (ncgpu_format_elliptic).  stat.txt's line is
   printed here from the device's statistics with the reference's own cart2ell,
   and collision.txt from the host's records, every line as display() prints
   it.  CM_buffer receives the copy's central body.  Returns 0 (nothing
   written) when the host must print this output itself: a cartesian value
   beyond the device formatter's range. */
static int gpu_display_device(void)
{
      static char *text = NULL;
      static unsigned long cap = 0;
      static double *yx = NULL, *F = NULL, *halk = NULL;
      static struct moonlet *hrec = NULL;
      static int *hidx = NULL;
      if (cap < ncgpu_format_cartesian_cap()) {  /* one pinned buffer for the whole run */
            if (text) {
                  ncgpu_host_unregister(text);
                  free(text);
            }
            cap = ncgpu_format_cartesian_cap();
            text = (char *)malloc(cap);
            if (text == NULL) {
                  fprintf(stderr, "Error : Can't allocate the output text buffer.\n");
                  abort();
            }
            gpu_check(ncgpu_host_register(text, cap), "host register");
      }
      if (write_elliptic_bool && yx == NULL) {  /* per body: atan2 arguments and results, listed bodies */
            const size_t nb = (size_t)N_max + 1;
            yx = (double *)malloc(2 * nb * sizeof(double));
            F = (double *)malloc(nb * sizeof(double));
            halk = (double *)malloc(6 * nb * sizeof(double));
            hrec = (struct moonlet *)malloc(nb * sizeof(struct moonlet));
            hidx = (int *)malloc(nb * sizeof(int));
            if (!yx || !F || !halk || !hrec || !hidx) {
                  fprintf(stderr, "Error : Can't allocate the elliptic output buffers.\n");
                  abort();
            }
            gpu_check(ncgpu_host_register(yx, 2 * nb * sizeof(double)), "host register");
            gpu_check(ncgpu_host_register(F, nb * sizeof(double)), "host register");
      }
      unsigned long lens[8];
      int st;
      if (write_cartesian_bool) {
            st = ncgpu_format_cartesian(text, cap, lens);
            if (st == NCGPU_E_UNSUPPORTED) return 0;
            gpu_check(st, "output text");
      }
      double stats[3];
      int idx[2];
      struct moonlet two[2];
      gpu_check(ncgpu_output_stats(stats, idx, (struct ncgpu_body *)&CM_buffer, (struct ncgpu_body *)two), "output stats");
      if (central_tides_bool || (J2_bool && J2_value == 0.)) gpu_check(ncgpu_get_sideral_omega(&SideralOmega), "sideral rotation");
      if (J2_bool) gpu_check(ncgpu_get_j2(&J2, NULL), "J2");  /* cart2ell reads it (src/structure.c:205-207) */

      int collision = collision_bool && write_collisions_bool ? 1 : 0;
      FILE *filestat = *files;
      FILE *out[8];   /* in the device's order: x y z vx vy vz mass radius */
      FILE *eout[6];  /* a lambda k h q p */
      if (write_cartesian_bool || write_elliptic_bool) {
            out[6] = *(files + 1 + collision);
            out[7] = *(files + 2 + collision);
      }
      if (write_cartesian_bool) {
            for (int f = 0; f < 6; f++) out[f] = *(files + 3 + collision + f);
            unsigned long pos = 0;
            for (int f = 0; f < 8; f++) {
                  fwrite(text + pos, 1, lens[f], out[f]);
                  pos += lens[f];
            }
      }

      typ total_mass = stats[0], M1 = stats[1], M2 = stats[2];
      typ mu, R1, R2, a1, a2, l1, l2, K1, K2, H1, H2, Q1, Q2, P1, P2, inner_fluid_disk_mass;
      typ alkhqp[6];
      mu = central_mass_bool ? CM_buffer.mass : M_unit;  mu += inner_fluid_disk_bool ? fluid_disk_Sigma*M_PI*(Rout*Rout - R_unit*R_unit) : 0.;  mu *= G;
      if (write_elliptic_bool) {
            const int first = write_cartesian_bool ? 9 : 3;
            for (int f = 0; f < 6; f++) eout[f] = *(files + first + collision + f);
            int nb = 0, nh = 0;
            gpu_check(ncgpu_elliptic_begin(mu, yx, 2ul * ((unsigned long)N_max + 1ul), &nb, hidx,
                                           (struct ncgpu_body *)hrec, N_max + 1, &nh), "elliptic elements");
            gpu_check(ncgpu_host_atan2(yx, F, nb), "atan2");
            for (int k = 0; k < nh; k++) cart2ell(hrec, k, halk + 6 * k, mu + G*hrec[k].mass);
            const int mr = write_cartesian_bool ? 0 : 1;  /* mass.txt and radius.txt, unless written above */
            st = ncgpu_format_elliptic(F, halk, nh, mr, text, cap, lens);
            if (st == NCGPU_E_UNSUPPORTED) {  /* a value beyond the formatter's range: print them here */
                  double *v = (double *)malloc(8 * ((size_t)nb + 1) * sizeof(double));
                  if (v == NULL) {
                        fprintf(stderr, "Error : Can't allocate the elliptic values.\n");
                        abort();
                  }
                  gpu_check(ncgpu_elliptic_values(v, 8ul * ((unsigned long)nb + 1ul)), "elliptic values");
                  for (int f = 0; f < 6 + 2 * mr; f++) {
                        FILE *o = f < 6 ? eout[f] : out[f];
                        for (int j = 0; j < nb; j++) fprintf(o, "%.14lf ", v[(size_t)f * nb + j]);
                  }
                  free(v);
            }
            else {
                  gpu_check(st, "elliptic text");
                  unsigned long pos = 0;
                  for (int f = 0; f < 6 + 2 * mr; f++) {
                        fwrite(text + pos, 1, lens[f], f < 6 ? eout[f] : out[f]);
                        pos += lens[f];
                  }
            }
      }
      if (how_many_moonlets == 0){
            M1 = 0.; M2 = 0.; R1 = 0.; R2 = 0.; a1 = 0.; a2 = 0.; l1 = 0.; l2 = 0.; K1 = 0.; K2 = 0.; H1 = 0.; H2 = 0.; Q1 = 0.; Q2 = 0.; P1 = 0.; P2 = 0.;
      }
      else if (how_many_moonlets == 1){
            M2 = 0.; R2 = 0.; a2 = 0.; l2 = 0.; K2 = 0.; H2 = 0.; Q2 = 0.; P2 = 0.;
            R1 = two[0].radius;
            cart2ell(two, 0, alkhqp, mu + G*M1);
            a1 = *alkhqp; l1 = alkhqp[1]; K1 = alkhqp[2]; H1 = alkhqp[3]; Q1 = alkhqp[4]; P1 = alkhqp[5];
      }
      else{
            R1 = two[0].radius;  R2 = two[1].radius;
            cart2ell(two, 0, alkhqp, mu + G*M1);
            a1 = *alkhqp; l1 = alkhqp[1]; K1 = alkhqp[2]; H1 = alkhqp[3]; Q1 = alkhqp[4]; P1 = alkhqp[5];
            cart2ell(two, 1, alkhqp, mu + G*M2);
            a2 = *alkhqp; l2 = alkhqp[1]; K2 = alkhqp[2]; H2 = alkhqp[3]; Q2 = alkhqp[4]; P2 = alkhqp[5];
      }
      fprintf(filestat, "%.14lf %d %d", time_elapsed + t_init, how_many_moonlets, collision_count);
      if (central_mass_bool) fprintf(filestat, " %.14lf", CM_buffer.mass);
      else fprintf(filestat, " %.1lf",  0.);
      fprintf(filestat, " %.14lf", total_mass);
      if (inner_fluid_disk_bool){
            inner_fluid_disk_mass = fluid_disk_Sigma*M_PI*(Rout*Rout - R_unit*R_unit);
            fprintf(filestat, " %.14lf %.14lf", inner_fluid_disk_mass, Rout);
      }
      else fprintf(filestat, " %.1lf %.1lf",  0., 0.);
      if (central_tides_bool || (J2_bool && J2_value == 0.)) fprintf(filestat, " %.14lf", SideralOmega);
      else fprintf(filestat, " %.1lf", 0.);
      fprintf(filestat, " %.14lf %.14lf %.14lf %.14lf %.14lf %.14lf %.14lf %.14lf %.14lf %.14lf %.14lf %.14lf %.14lf %.14lf %.14lf %.14lf",
      M1, M2, R1, R2, a1, a2, l1, l2, K1, K2, H1, H2, Q1, Q2, P1, P2);
      fprintf(filestat, "\n");
      if (write_cartesian_bool) for (int f = 0; f < 6; f++) fprintf(out[f], "\n");
      if (write_elliptic_bool) for (int f = 0; f < 6; f++) fprintf(eout[f], "\n");
      if (write_cartesian_bool || write_elliptic_bool) {
            fprintf(out[7], "\n");  /* radius.txt, then mass.txt, as display() ends them */
            fprintf(out[6], "\n");
      }
      if (collision){
            FILE *filecol = *(files + 1);
            for (int p = 0; p < indexCollision; p ++){
                  struct collisionData *cd = collisionDatas + p;
                  fprintf(filecol, "%.14lf %.14lf %.14lf %.14lf %.14lf %.14lf %.14lf %.14lf\n", cd->time, cd->m1, cd->m2,
                          cd->R1, cd->R2, cd->DeltaV, cd->impact_angle, cd->m_tilde);
            }
            indexCollision = 0;
      }
      return 1;
}

static int gpu_collide_brute(double t_now)
{
      int n = 0;
      gpu_check(ncgpu_set_timestep(timestep), "timestep");
      gpu_check(ncgpu_collide_brute(&n), "brute_force");
      collision_count += n;
      gpu_collision_records(t_now);
      return n;
}

/* end_of_timestep's printout at a progress step (src/rk4.c:225-333) from the
   device's statistics (total mass, the two most massive bodies, the
   barycentre, largest_id before tidy_up), the host's counters and the
   reference's own cart2ell, instead of a copy of the whole state; CM and
   CM_buffer as the reference leaves them. */
static void gpu_progress_printout(void)
{
      typ stats[3], com[6], alkhqp[6];
      int idx[2], lid = 0, lid_printed = 0;
      struct moonlet two[2];
      gpu_check(ncgpu_output_stats(stats, idx, (struct ncgpu_body *)&CM, (struct ncgpu_body *)two), "stats");
      gpu_check(ncgpu_total_momentum(com), "total_momentum");
      gpu_check(ncgpu_get_largest_id(&lid, &lid_printed), "largest_id");
      if (central_tides_bool || (J2_bool && J2_value == 0.))
            gpu_check(ncgpu_get_sideral_omega(&SideralOmega), "sideral rotation");
      if (J2_bool) {  /* the printout precedes end_of_timestep's J2 update (src/rk4.c:459-463) */
            typ j2_now = 0.;
            gpu_check(ncgpu_get_j2(&j2_now, &J2), "J2");
      }
      if (fragmentation_bool) {  /* the outcome shares (src/rk4.c:244-247) */
            int fc[4];
            gpu_check(ncgpu_fragment_counts(fc), "fragment counts");
            merger_count = fc[0];
            super_catastrophic_count = fc[1];
            half_fragmentation_count = fc[2];
            full_fragmentation_count = fc[3];
      }
      typ total_mass = stats[0], M1 = stats[1], M2 = stats[2];
      typ R1, R2, a1, a2, e1, e2, I1, I2, l1, l2, o1, o2, O1, O2;
      if (central_mass_bool){
            CM_buffer = CM;
            CM_buffer.x -= .5*timestep*CM_buffer.vx;  CM_buffer.y -= .5*timestep*CM_buffer.vy;  CM_buffer.z -= .5*timestep*CM_buffer.vz;
      }
      if (collision_bool){
            printf("                  N = %d  |  Collisions = %d  |  t = %.13lf   (largest id in the body array = %d)\n",
            how_many_moonlets, collision_count, t_init + time_elapsed, lid_printed);
      }
      else{
            printf("                  N = %d  |  t = %.13lf   (largest id in the body array = %d)\n", how_many_moonlets, t_init + time_elapsed, lid_printed);
      }
      if (collision_bool && fragmentation_bool && collision_count != 0){
            typ cll = (typ) collision_count;
            typ mrg = 100.*((typ) merger_count)/cll;
            typ spc = 100.*((typ) super_catastrophic_count)/cll;
            typ hfr = 100.*((typ) half_fragmentation_count)/cll;
            typ ffr = 100.*((typ) full_fragmentation_count)/cll;
            printf("                  Merger = %.2lf %% | Super-catastrophic = %.2lf %% | Partially fragmented = %.2lf %% | Fully fragmented = %.2lf %%\n",
            mrg, spc, hfr, ffr);
      }
      if (central_mass_bool){
            printf("                  Central mass = %.8lf,  Bodies mass = %.8lf\n", CM.mass, total_mass);
      }
      else{
            printf("                  Bodies total mass = %.8lf\n", total_mass);
      }
      typ mu = central_mass_bool ? CM.mass : M_unit;  mu *= G;
      if (how_many_moonlets > 1){
            typ vp1, vp2;
            struct moonlet mlt1 = {two[0].x, two[0].y, two[0].z, two[0].vx, two[0].vy, two[0].vz, 0., 0.};
            struct moonlet mlt2 = {two[1].x, two[1].y, two[1].z, two[1].vx, two[1].vy, two[1].vz, 0., 0.};
            mlt1.x -= .5*timestep*mlt1.vx;  mlt1.y -= .5*timestep*mlt1.vy;  mlt1.z -= .5*timestep*mlt1.vz;
            mlt2.x -= .5*timestep*mlt2.vx;  mlt2.y -= .5*timestep*mlt2.vy;  mlt2.z -= .5*timestep*mlt2.vz;
            R1  = two[0].radius;  R2 = two[1].radius;
            cart2ell(&mlt1, 0, alkhqp, mu + G*M1);
            a1  = *alkhqp; e1 = sqrt(alkhqp[2]*alkhqp[2] + alkhqp[3]*alkhqp[3]); I1 = 360.*asin(sqrt(alkhqp[4]*alkhqp[4] + alkhqp[5]*alkhqp[5]))/M_PI;
            vp1 = 180.*atan2(alkhqp[3], alkhqp[2])/M_PI;
            l1  = 180.*alkhqp[1]/M_PI - vp1; O1 = 180.*atan2(alkhqp[5], alkhqp[4])/M_PI; o1 = vp1 - O1;
            cart2ell(&mlt2, 0, alkhqp, mu + G*M2);
            a2  = *alkhqp; e2 = sqrt(alkhqp[2]*alkhqp[2] + alkhqp[3]*alkhqp[3]); I2 = 360.*asin(sqrt(alkhqp[4]*alkhqp[4] + alkhqp[5]*alkhqp[5]))/M_PI;
            vp2 = 180.*atan2(alkhqp[3], alkhqp[2])/M_PI;
            l2  = 180.*alkhqp[1]/M_PI - vp2; O2 = 180.*atan2(alkhqp[5], alkhqp[4])/M_PI; o2 = vp2 - O2;
            printf("                  Most massive : (m, R; a, e, i; M, o, O) = (%.7lf, %.4lf; %.3lf, %.3lf, %.3lf°; %.2lf°, %.2lf°, %.2lf°)\n",
            M1, R1, a1, e1, I1, l1, o1, O1);
            printf("                  Second most  : (m, R; a, e, i; M, o, O) = (%.7lf, %.4lf; %.3lf, %.3lf, %.3lf°; %.2lf°, %.2lf°, %.2lf°)\n",
            M2, R2, a2, e2, I2, l2, o2, O2);
      }
      else if (how_many_moonlets == 1){
            typ vp1;
            struct moonlet mlt1 = {two[0].x, two[0].y, two[0].z, two[0].vx, two[0].vy, two[0].vz, 0., 0.};
            mlt1.x -= .5*timestep*mlt1.vx;  mlt1.y -= .5*timestep*mlt1.vy;  mlt1.z -= .5*timestep*mlt1.vz;
            R1  = two[0].radius;
            cart2ell(&mlt1, 0, alkhqp, mu + G*M1);
            a1  = *alkhqp; e1 = sqrt(alkhqp[2]*alkhqp[2] + alkhqp[3]*alkhqp[3]); I1 = 360.*asin(sqrt(alkhqp[4]*alkhqp[4] + alkhqp[5]*alkhqp[5]))/M_PI;
            vp1 = 180.*atan2(alkhqp[3], alkhqp[2])/M_PI;
            l1  = 180.*alkhqp[1]/M_PI - vp1; O1 = 180.*atan2(alkhqp[5], alkhqp[4])/M_PI; o1 = vp1 - O1;
            printf("                  Most massive : (m, R; a, e, i; M, o, O) = (%.7lf, %.4lf; %.3lf, %.3lf, %.3lf°; %.2lf°, %.2lf°, %.2lf°)\n",
            M1, R1, a1, e1, I1, l1, o1, O1);
      }
      if (central_tides_bool){
            printf("                  Sideral rotation = %.13lf\n", SideralOmega);
      }
      printf("                  COM = (%.9lf, %.9lf,  %.9lf,  %.9lf,  %.9lf,  %.9lf)\n", com[0], com[1], com[2], com[3], com[4], com[5]);
      largest_id = lid;
}

/* end of a step on the device, then the host's share of end_of_timestep
   (src/rk4.c:130-473): how_many_moonlets, at a progress step the printout,
   in mesh mode gamma (src/rk4.c:356-381) and the brute-force switch
   (src/rk4.c:384-389).  The fluid-body J2 the device keeps itself; the host's
   copy is refreshed when the host needs it (gpu_pull). */
static void gpu_end_of_timestep(struct moonlet *moonlets, int progressed, long total_nb)
{
      int hm = 0;
      gpu_check(ncgpu_end_of_timestep(&hm), "end_of_timestep");
      how_many_moonlets = hm;
      first_passage = 1;
      if (progressed) gpu_progress_printout();
#if mesh_bool
      if ((collision_bool || mutual_bool) && !force_naive_bool) {
            how_many_pairs = 0;
            average_neighbours = 2.0 * ((typ)total_nb) / ((typ)how_many_moonlets);
            gam *= pow(how_many_neighbours / average_neighbours, 1.0 / 3.0);
            if (gam < gam_min) gam = gam_min;
            collision_cube = gam * ((typ)collision_cube_cells);
            if (progressed) {
                  printf("                  average number of neighbours = %.3lf\n", average_neighbours);
                  printf("                  gamma = %.6lf\n", gam);
            }
            how_many_modified = 0;
            how_many_big = 0;
            how_many_small = 0;
            total_neighbours = 0;
      }
#endif
      if (!brute_force_bool && !force_naive_bool && how_many_moonlets < switch_to_brute_force)
            force_naive_bool = 1;
      else if (!brute_force_bool && force_naive_bool && how_many_moonlets > switch_to_brute_force)
            force_naive_bool = 0;
      if (J2_bool) gpu_check(ncgpu_get_j2(&J2, NULL), "J2");  /* after end_of_timestep's update */
      (void)moonlets;  /* the host copy is refreshed only where the host uses it (gpu_pull) */
      gpu_check(ncgpu_set_force_naive(force_naive_bool), "force_naive");
}

static void gpu_start(struct moonlet **moonlets, struct moonlet **buffer)
{
      struct ncgpu_params p;
      gpu_supported();
      *moonlets = populate();
      *buffer = (struct moonlet *)malloc(N_max * sizeof(struct moonlet));
      if (*buffer == NULL) {
            fprintf(stderr, "Error : Can't allocate buffer for array of bodies.\n");
            abort();
      }
      gpu_params(&p);
      gpu_check(ncgpu_init(N_max, &p), "init");
      gpu_check(ncgpu_host_register(*moonlets, sizeof(struct moonlet) * (unsigned long)N_max), "host register");
      gpu_upload(*moonlets);
      gpu_check(ncgpu_set_timestep(timestep), "timestep");
      gpu_check(ncgpu_set_force_naive(force_naive_bool), "force_naive");
}

/* The last output without a state copy (write_to_files_bool, no resume
   files): the final half backward drift or kick already ran on a device
   snapshot, which is printed here.  Returns 0 when the host must print it. */
static int gpu_final_display_device(struct moonlet *buffer)
{
      int done = gpu_display_device();
      if (!done) {
            gpu_snapshot_pull(buffer);
            display(buffer);
      }
      gpu_check(ncgpu_snapshot_end(), "snapshot");
      return 1;
}

static void gpu_stop(struct moonlet *moonlets, struct moonlet *buffer, bigint iter, int displayed)
{
      if (write_to_files_bool && !displayed) display(moonlets);
      if (resume_simulation_bool) {
            resume(moonlets);
            resumeFile();
      }
      printf("progress = %.1lf %%\n", 100.0);
      printf("total number of timestep performed : %ld\n", iter);
      ncgpu_host_unregister(moonlets);
      ncgpu_finalize();
      free(moonlets);
      free(buffer);
}

/* integration_brute_force_SABA1 (src/rk4.c:840-954) */
void ncgpu_integration_brute_force_SABA1(typ t)
{
      struct moonlet *moonlets, *moonlet_buffer;
      bigint iter = 0;
      int progressed = 0, j;
      typ progress = 0.0, previous_progress = 0.0;
      gpu_start(&moonlets, &moonlet_buffer);
      printf("progress = %.1lf %%\n", 0.0);
      if (write_to_files_bool) {
            readme();
            if (central_mass_bool) CM_buffer = CM;
            if (!gpu_display_device()) display(moonlets);  /* the uploaded state, formatted on the device */
      }
      if (t > 0.0) {  /* half drift */
            timestep /= 2.0;
            if (collision_bool) gpu_collide_brute(t_init + time_elapsed);
            gpu_check(ncgpu_set_timestep(timestep), "timestep");
            gpu_check(ncgpu_drift(), "drift");
            timestep *= 2.0;
            gpu_check(ncgpu_set_timestep(timestep), "timestep");
      }
      while (time_elapsed < t) {
            progressed = 0;
            if (write_to_files_bool && iter % output_step == 0 && iter > 0) {
                  /* the half backward drift of a copy, printed (src/rk4.c:881-890), on the device */
                  gpu_check(ncgpu_snapshot_begin(), "snapshot");
                  gpu_check(ncgpu_set_timestep(timestep / -2.0), "timestep");
                  gpu_check(ncgpu_drift(), "drift");
                  if (!gpu_display_device()) {
                        gpu_snapshot_pull(moonlet_buffer);
                        display(moonlet_buffer);
                  }
                  gpu_check(ncgpu_snapshot_end(), "snapshot");
                  gpu_check(ncgpu_set_timestep(timestep), "timestep");
            }
            gpu_check(ncgpu_kick(), "kick");
            time_elapsed += .5 * timestep;
            if (collision_bool) gpu_collide_brute(t_init + time_elapsed);
            gpu_check(ncgpu_drift(), "drift");
            iter++;
            time_elapsed += .5 * timestep;
            progress = time_elapsed / t;
            if (progress - previous_progress > .001) {
                  previous_progress = progress;
                  printf("progress = %.1lf %%\n", 100. * progress);
                  progressed = 1;
            }
            gpu_end_of_timestep(moonlets, progressed, 0);
      }
      if (write_to_files_bool && !resume_simulation_bool) {  /* the last output from a device snapshot */
            gpu_check(ncgpu_snapshot_begin(), "snapshot");
            if (t > 0.) {  /* half backward drift of the final output */
                  gpu_check(ncgpu_set_timestep(timestep / -2.), "timestep");
                  gpu_check(ncgpu_drift(), "drift");
            }
            gpu_stop(moonlets, moonlet_buffer, iter, gpu_final_display_device(moonlet_buffer));
            return;
      }
      /* the final state (CM is the state's), then its half backward drift on a
         device copy: the bodies and CM_buffer come from the copy */
      gpu_pull(moonlets);
      if (central_mass_bool) CM_buffer = CM;
      if (t > 0.) {
            gpu_check(ncgpu_snapshot_begin(), "snapshot");
            gpu_check(ncgpu_set_timestep(timestep / -2.), "timestep");
            gpu_check(ncgpu_drift(), "drift");
            gpu_snapshot_pull(moonlets);
            gpu_check(ncgpu_snapshot_end(), "snapshot");
      }
      gpu_stop(moonlets, moonlet_buffer, iter, 0);
}

#if mesh_bool
/* three largest to slots 0-2, one mesh pass; returns total_neighbours */
static long gpu_mesh_pass(int with_collisions)
{
      int np = 0, ne = 0;
      long tn = 0;
      gpu_check(ncgpu_three_largest(NULL), "three_largest");
      gpu_check(ncgpu_set_timestep(timestep), "timestep");
      gpu_check(ncgpu_mesh(gam, with_collisions, &np, &ne, &tn), "mesh");
      if (with_collisions) {
            collision_count += ne;
            gpu_collision_records(t_init + time_elapsed);
      }
      return tn;
}

/* integration_mesh (src/rk4.c:662-837) */
void ncgpu_integration_mesh(typ t)
{
      struct moonlet *moonlets, *moonlet_buffer;
      bigint iter = 0;
      int progressed = 0, j, index;
      typ progress = 0.0, previous_progress = 0.0;
      long tn;
      gpu_start(&moonlets, &moonlet_buffer);
      printf("progress = %.1lf %%\n", 0.0);
      if (write_to_files_bool) {
            readme();
            if (central_mass_bool) CM_buffer = CM;
            if (!gpu_display_device()) display(moonlets);  /* the uploaded state, formatted on the device */
      }
      if (t > 0.0) {  /* half kick */
            timestep /= 2.0;
            tn = gpu_mesh_pass(0);
            gpu_check(ncgpu_kick(), "kick");
            gpu_check(ncgpu_mesh_reset(), "mesh reset");
            timestep *= 2.0;
            gpu_check(ncgpu_set_timestep(timestep), "timestep");
            average_neighbours = 2.0 * ((typ)tn) / ((typ)how_many_moonlets);
            gam *= pow(how_many_neighbours / average_neighbours, 1.0 / 3.0);
            if (gam < gam_min) gam = gam_min;
            collision_cube = gam * ((typ)collision_cube_cells);
            how_many_pairs = 0;
            total_neighbours = 0;
      }
      while (time_elapsed < t) {
            progressed = 0;
            if (write_to_files_bool && iter % output_step == 0 && iter > 0) {
                  /* the half backward kick of a copy, printed (src/rk4.c:740-757), on the
                     device: the copy shares exists[], the free slots and SideralOmega
                     with the bodies, as the reference's globals do */
                  gpu_check(ncgpu_snapshot_begin(), "snapshot");
                  gpu_check(ncgpu_set_timestep(timestep / -2.0), "timestep");
                  if (!force_naive_bool) {
                        int np = 0, ne = 0;
                        long tn0 = 0;
                        gpu_check(ncgpu_three_largest(NULL), "three_largest");
                        gpu_check(ncgpu_mesh(gam, 0, &np, &ne, &tn0), "mesh");  /* get_neighbours_mesh */
                  }
                  gpu_check(ncgpu_kick(), "kick");
                  if (!gpu_display_device()) {
                        gpu_snapshot_pull(moonlet_buffer);
                        display(moonlet_buffer);
                  }
                  gpu_check(ncgpu_snapshot_end(), "snapshot");
                  if (!force_naive_bool) {
                        gpu_check(ncgpu_mesh_reset(), "mesh reset");
                        how_many_pairs = 0;
                        how_many_modified = 0;
                        total_neighbours = 0;
                  }
                  gpu_check(ncgpu_set_timestep(timestep), "timestep");
            }
            tn = 0;
            if (collision_bool) {
                  if (force_naive_bool) gpu_collide_brute(t_init + time_elapsed);
                  else tn = gpu_mesh_pass(1);
            }
            gpu_check(ncgpu_set_timestep(timestep), "timestep");
            gpu_check(ncgpu_drift(), "drift");
            time_elapsed += 0.5 * timestep;
            if (!collision_bool && !force_naive_bool) tn = gpu_mesh_pass(0);
            gpu_check(ncgpu_kick(), "kick");
            iter++;
            time_elapsed += 0.5 * timestep;
            progress = time_elapsed / t;
            if (progress - previous_progress > 0.001) {
                  previous_progress = progress;
                  printf("progress = %.1lf %%\n", 100.0 * progress);
                  progressed = 1;
            }
            gpu_end_of_timestep(moonlets, progressed, tn);
      }
      if (write_to_files_bool && !resume_simulation_bool) {  /* the last output from a device snapshot */
            gpu_check(ncgpu_snapshot_begin(), "snapshot");
            if (t > 0.0) {  /* half backward kick of the final state */
                  gpu_check(ncgpu_set_timestep(timestep / -2.0), "timestep");
                  if (!force_naive_bool) {
                        int np = 0, ne = 0;
                        long tn0 = 0;
                        gpu_check(ncgpu_three_largest(NULL), "three_largest");
                        gpu_check(ncgpu_mesh(gam, 0, &np, &ne, &tn0), "mesh");
                  }
                  gpu_check(ncgpu_kick(), "kick");
            }
            gpu_stop(moonlets, moonlet_buffer, iter, gpu_final_display_device(moonlet_buffer));
            return;
      }
      /* the final state (CM is the state's), then its half backward kick on a
         device copy: the three largest bodies' reordering, the neighbours and
         the gravity of the copy, whose bodies and CM_buffer the host gets */
      gpu_pull(moonlets);
      if (central_mass_bool) CM_buffer = CM;
      if (t > 0.0) {
            gpu_check(ncgpu_snapshot_begin(), "snapshot");
            gpu_check(ncgpu_set_timestep(timestep / -2.0), "timestep");
            if (!force_naive_bool) {
                  int np = 0, ne = 0;
                  long tn0 = 0;
                  gpu_check(ncgpu_three_largest(NULL), "three_largest");
                  gpu_check(ncgpu_mesh(gam, 0, &np, &ne, &tn0), "mesh");
            }
            gpu_check(ncgpu_kick(), "kick");
            gpu_snapshot_pull(moonlets);
            gpu_check(ncgpu_snapshot_end(), "snapshot");
      }
      gpu_stop(moonlets, moonlet_buffer, iter, 0);
}
#endif
