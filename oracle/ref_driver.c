/*
 * Test-infrastructure driver linked against the reference's own, unmodified
 * C sources (compiled by oracle/ref_build.py into oracle/_ref/<profile>/).
 * It exposes the hot-path functions of the reference through the small
 * "orc_*" C API that the parity tests load with ctypes.  Nothing here is
 * part of the product; it only sets the reference's globals, calls its
 * functions and copies results out.
 *
 * Reference functions called (all paths relative to the reference project):
 *   vector_field           src/physics.c:63
 *   kick / drift           src/rk4.c:68, src/rk4.c:109
 *   end_of_timestep        src/rk4.c:130
 *   brute_force            src/collision.c:425
 *   mesh                   src/collision.c:324
 *   get_neighbours_mesh    src/physics.c:1094
 *   three_largest_*        src/structure.c:914, src/structure.c:1005
 *   collision_treatment    src/physics.c:1043 (wrapped with -Wl,--wrap to log events)
 *   fragmentation counters src/structure.h:148-151
 *   falcON tree            src/ffm.c (tables src/main.c:118-125, build
 *                          src/rk4.c:576-586, release src/rk4.c:337-346)
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "parameters.h"
#include "structure.h"
#include "physics.h"
#include "collision.h"
#include "rk4.h"
#include "ffm.h"

static struct moonlet *B = NULL;    /* the body array handed to the reference */
static int *ev_log = NULL;          /* (a, b, type) per collision_treatment call */
static int ev_n = 0, ev_cap = 0;

void __real_collision_treatment(struct moonlet *moonlets, int a, int b, int type_of_collision);

void __wrap_collision_treatment(struct moonlet *moonlets, int a, int b, int type_of_collision)
{
      if (ev_n >= ev_cap) {
            ev_cap = ev_cap ? 2 * ev_cap : 4096;
            ev_log = (int *)realloc(ev_log, 3 * sizeof(int) * (size_t)ev_cap);
      }
      ev_log[3 * ev_n] = a;
      ev_log[3 * ev_n + 1] = b;
      ev_log[3 * ev_n + 2] = type_of_collision;
      ev_n++;
      __real_collision_treatment(moonlets, a, b, type_of_collision);
}

int orc_n_max(void) { return N_max; }
int orc_cells(void)
{
#if mesh_bool
      return collision_cube_cells;
#else
      return 0;
#endif
}

int orc_init(void)
{
      variable_initialization();
      array_initialization();
      B = (struct moonlet *)calloc((size_t)N_max, sizeof(struct moonlet));
      return B == NULL ? -1 : 0;
}

/* bodies: 8 doubles per slot for slots 0..lid; ex: exists flag per slot;
   cm: 8 doubles (central mass); dt: timestep; g: mesh size gamma (mesh only) */
void orc_set_state(int lid, const double *bodies, const int *ex, const double *cm, double dt, double g)
{
      int j;
      largest_id = lid;
      memcpy(B, bodies, sizeof(struct moonlet) * (size_t)(lid + 1));
      for (j = 0; j < N_max; j++) exists[j] = j <= lid ? ex[j] : 0;
      memcpy(&CM, cm, sizeof(struct moonlet));
      timestep = dt;
      how_many_free = 0;
      how_many_moonlets = 0;
      for (j = 0; j <= lid; j++) how_many_moonlets += ex[j] ? 1 : 0;
      need_to_reduce_COM_bool = 0;
      /* the central body's rotation and the J2 in force for this central
         mass, as variable_initialization sets them (src/structure.c:506-507) */
      SideralOmega = 2. * M_PI / Tearth;
#if J2_bool
      J2 = J2_value == 0. ? 0.5 * SideralOmega * SideralOmega * R_unit * R_unit * R_unit / (G * CM.mass) : J2_value;
#endif
#if mesh_bool
      gam = g;
      collision_cube = gam * ((typ)collision_cube_cells);
#else
      (void)g;
#endif
#if collision_bool
      for (j = 0; j < N_max; j++) did_collide[j] = 0;
#endif
}

/* free-index stack (src/structure.c:849-878), for runs that recycle slots */
void orc_set_free(int n, const int *idx)
{
      int j;
      for (j = 0; j < n; j++) free_indexes[j] = idx[j];
      how_many_free = n;
}

int orc_get_state(double *bodies, int *ex, double *cm, double *scalars)
{
      int j;
      memcpy(bodies, B, sizeof(struct moonlet) * (size_t)(largest_id + 1));
      for (j = 0; j <= largest_id; j++) ex[j] = exists[j];
      memcpy(cm, &CM, sizeof(struct moonlet));
      if (scalars) {
            scalars[0] = timestep;
#if mesh_bool
            scalars[1] = gam;
#else
            scalars[1] = 0.;
#endif
            scalars[2] = (double)how_many_moonlets;
            scalars[3] = (double)collision_count;
            scalars[4] = time_elapsed;
      }
      return largest_id;
}

/* One force evaluation, exactly as kick() prepares it (src/rk4.c:76-85):
   existing bodies are copied into xx, then vector_field(xx) runs.  acc gets
   3 doubles per slot 0..largest_id; cm_acc the back-reaction on the central mass. */
void orc_vector_field(double *acc, double *cm_acc)
{
      int j;
      for (j = 0; j <= largest_id; j++)
            if (exists[j]) xx[j] = B[j];
      vector_field(xx);
      for (j = 0; j <= largest_id; j++) {
            acc[3 * j] = exists[j] ? xx[j].vx : 0.;
            acc[3 * j + 1] = exists[j] ? xx[j].vy : 0.;
            acc[3 * j + 2] = exists[j] ? xx[j].vz : 0.;
      }
      cm_acc[0] = CM_acc[0];
      cm_acc[1] = CM_acc[1];
      cm_acc[2] = CM_acc[2];
}

/* falcON: the multipole index tables main() fills once (src/main.c:118-125). */
void orc_tree_tables(void)
{
      k_from_s2s3_init();
      s1s2s3_from_kn_init();
      s2s3_from_k_init();
      k_from_ijklmn_init();
      ijklmn_from_kn_init();
      perm_from_kn_init();
      q1fromq2q3_init();
}

/* The tree of the current state, as the tree driver builds it before its kick
   (src/rk4.c:576-586); vector_field then runs falcON on it.  Returns the
   number of cells. */
int orc_tree_build(void)
{
      struct boxdot *root = root_cell(B);
      FlatTree = flattree_init(root);
      clear_boxdot(&root);
      com_flattree(FlatTree, B);
      Mtot = FlatTree->M0;
      rmax_flattree(FlatTree, B);
      rcrit_flattree(FlatTree);
      tensor_initialization(FlatTree);
#if expansion_order > 2
      multipole_flattree(FlatTree, B);
#endif
      return cell_id;
}

/* The next tree takes the bodies in slot order, as the first tree of a run
   does (IndexPeanoHilbertOrder at its initial 0); every later tree takes them
   in the previous tree's Peano-Hilbert order first (src/ffm.c:350-361,
   421-479), which changes the order of the sums in its leaves. */
void orc_tree_slot_order(void) { IndexPeanoHilbertOrder = 0; }

/* Releases the tree as end_of_timestep does (src/rk4.c:337-346). */
void orc_tree_free(void)
{
      int j;
      if (FlatTree == NULL) return;
      for (j = 0; j < cell_id; j++) {
            free((FlatTree + j)->dots);
            (FlatTree + j)->dots = NULL;
      }
      free(FlatTree);
      FlatTree = NULL;
      how_many_cells = 0;
      cell_id = 0;
}

void orc_kick(void) { kick(B, &CM, vector_field); }
void orc_drift(void) { drift(B, &CM); }
void orc_set_timestep(double dt) { timestep = dt; }
double orc_get_sideral_omega(void) { return SideralOmega; }
void orc_set_sideral_omega(double w) { SideralOmega = w; }
void orc_end_of_timestep(void) { end_of_timestep(B, 0); }

void orc_events_reset(void) { ev_n = 0; }

/* merger, super-catastrophic, partial and full fragmentation counts */
void orc_frag_counts(int *out)
{
      out[0] = merger_count;
      out[1] = super_catastrophic_count;
      out[2] = half_fragmentation_count;
      out[3] = full_fragmentation_count;
}
void orc_frag_counts_reset(void)
{
      merger_count = super_catastrophic_count = half_fragmentation_count = full_fragmentation_count = 0;
}
int orc_events(int *out, int cap)
{
      int n = ev_n < cap ? ev_n : cap;
      memcpy(out, ev_log, 3 * sizeof(int) * (size_t)n);
      return ev_n;
}

#if collision_bool
void orc_brute_force(void) { brute_force(B); }
#endif

#if mesh_bool
void orc_three_largest(int *idx)
{
      three_largest_moonlets(B);
      three_largest_three_first(B);
      idx[0] = three_largest_indexes[0];
      idx[1] = three_largest_indexes[1];
      idx[2] = three_largest_indexes[2];
}
#if collision_bool
void orc_mesh(void) { mesh(B); }
#endif
void orc_get_neighbours_mesh(void) { get_neighbours_mesh(B); }
int orc_pairs(int *out, int cap)
{
      int j, n = how_many_pairs < cap ? how_many_pairs : cap;
      for (j = 0; j < n; j++) {
            out[2 * j] = pairs[j].fst;
            out[2 * j + 1] = pairs[j].snd;
      }
      return how_many_pairs;
}
long orc_total_neighbours(void) { return (long)total_neighbours; }
void orc_mesh_counts(int *out)
{
      out[0] = how_many_small;
      out[1] = how_many_big;
      out[2] = how_many_modified;
}
/* Clears the hash table and the per-step mesh counters, the way the mesh
   driver does after a half kick (src/rk4.c:704-717), without touching gamma. */
void orc_mesh_reset(void)
{
      int j;
      for (j = 0; j < how_many_modified; j++) clear_chain(hash + modified_cells[j]);
      how_many_pairs = 0;
      how_many_modified = 0;
      total_neighbours = 0;
      how_many_big = 0;
      how_many_small = 0;
}
#endif

/* One iteration of the brute-force integrator loop (src/rk4.c:906-921),
   without output: kick, collisions, drift, end_of_timestep. */
void orc_step_brute_force(void)
{
      kick(B, &CM, vector_field);
      time_elapsed += .5 * timestep;
#if collision_bool && brute_force_bool
      brute_force(B);
#endif
      drift(B, &CM);
      time_elapsed += .5 * timestep;
      end_of_timestep(B, 0);
}

#if mesh_bool
/* One iteration of the mesh integrator loop (src/rk4.c:760-790), without output. */
void orc_step_mesh(void)
{
#if collision_bool
      if (force_naive_bool) {
            brute_force(B);
      } else {
            three_largest_moonlets(B);
            three_largest_three_first(B);
            mesh(B);
      }
#endif
      drift(B, &CM);
      time_elapsed += 0.5 * timestep;
      if (!collision_bool && !force_naive_bool) {
            three_largest_moonlets(B);
            three_largest_three_first(B);
            get_neighbours_mesh(B);
      }
      kick(B, &CM, vector_field);
      time_elapsed += 0.5 * timestep;
      end_of_timestep(B, 0);
}
#endif

/* cart2ell (src/structure.c:172-284) of one record with the central body cm
   as CM_buffer and the J2 in force j2 (the global J2 it reads), as display()
   calls it; the reference prints its warnings to stdout. */
void orc_cart2ell(const double *rec, const double *cm, double j2, double mu, double *alkhqp)
{
      struct moonlet m;
      memcpy(&m, rec, sizeof m);
      memcpy(&CM_buffer, cm, sizeof CM_buffer);
      J2 = j2;
      cart2ell(&m, 0, alkhqp, mu);
      fflush(stdout);
}
