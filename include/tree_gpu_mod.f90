! tree_gpu_mod.f90 -- ISO_C_BINDING interface of libtree_b200.so for the
! Fortran driver of TREE (main.f90).  Declares every entry point of
! tree_gpu.h with BIND(C).  TYPE(PT) (data.f90:47-50) has no interoperable
! layout, so the caller packs positions, velocities and forces into
! REAL(C_DOUBLE) arrays of 3*N (x1,y1,z1,x2,...), the layout TYPE(GS) holds.
!
! Call-site changes in main.f90:
!   * Vinit / Vinit_REST (main.f90:777, 821): tree_gpu_set_state after the
!     velocities are drawn or read;
!   * the loop body (main.f90:125-131), or the whole loop with its TEMPORAL and
!     RDF cadence (main.f90:123-160): tree_gpu_step / tree_gpu_run;
!   * Restart steps: tree_gpu_get_state, then unpack into qel/qion.
! RDF_ei / RDF_ii are INTEGER in the reference (data.f90:139): pass
! INTEGER(C_INT64_T) copies of TREE_GPU_RDF_BINS entries and add them back.
MODULE TREE_GPU_MOD
  USE ISO_C_BINDING
  IMPLICIT NONE

  INTEGER(C_INT), PARAMETER :: TREE_GPU_OK = 0, TREE_GPU_ERR_ARG = -1, &
       TREE_GPU_ERR_DEPTH = -2, TREE_GPU_ERR_NONFINITE = -3, &
       TREE_GPU_ERR_CAPACITY = -4, TREE_GPU_ERR_CUDA = -5, &
       TREE_GPU_ERR_WALK = -6, TREE_GPU_ERR_STATE = -7
  INTEGER(C_INT32_T), PARAMETER :: TREE_GPU_PHYS_REF = 0, TREE_GPU_PHYS_KELBG = 1
  INTEGER(C_INT32_T), PARAMETER :: TREE_GPU_PREC_FP64 = 0, TREE_GPU_PREC_MIXED = 1
  INTEGER(C_INT32_T), PARAMETER :: TREE_GPU_MAC_FIXED = 0, TREE_GPU_MAC_LEARNED = 1
  INTEGER, PARAMETER :: TREE_GPU_RDF_BINS = 10001
  INTEGER, PARAMETER :: TREE_GPU_MLP_PARAMS = 5313, TREE_GPU_MLP_STATS = 72

  TYPE, BIND(C) :: tree_gpu_params
     REAL(C_DOUBLE) :: theta      ! param%sd_ratio
     REAL(C_DOUBLE) :: rs         ! param%rs (um)
     REAL(C_DOUBLE) :: te         ! electron temperature for lambda_ij (K)
     REAL(C_DOUBLE) :: xm_el      ! param%xm(1) (amu)
     REAL(C_DOUBLE) :: xm_ion     ! param%xm(2) (amu)
     REAL(C_DOUBLE) :: dx_ei      ! NS%dx_ei (um)
     REAL(C_DOUBLE) :: dx_ii      ! NS%dx_ii (um)
     INTEGER(C_INT32_T) :: physics, precision, mac, group
  END TYPE tree_gpu_params

  TYPE, BIND(C) :: tree_gpu_diag
     REAL(C_DOUBLE) :: epot_e, epot_i, mv2_el, mv2_ion, rad_el, rad_ion
     INTEGER(C_INT64_T) :: steps_done
  END TYPE tree_gpu_diag

  TYPE, BIND(C) :: tree_gpu_sample
     INTEGER(C_INT64_T) :: nloop
     REAL(C_DOUBLE) :: epot_e, epot_i, mv2_el, mv2_ion, rad_el, rad_ion
  END TYPE tree_gpu_sample

  TYPE, BIND(C) :: tree_gpu_timing
     REAL(C_DOUBLE) :: ms_build, ms_walk, ms_kdk, ms_total
     INTEGER(C_INT64_T) :: n_m2p, n_p2p, n_nodes, calls, launches, &
          n_mac_net, n_mac_fallback, n_m2p_total, n_p2p_total, &
          n_mac_net_total, n_local, n_local_total
  END TYPE tree_gpu_timing

  INTERFACE
     INTEGER(C_INT) FUNCTION tree_gpu_create(p, n_el, n_ion, h) BIND(C)
       IMPORT :: C_INT, C_INT64_T, C_PTR, tree_gpu_params
       TYPE(tree_gpu_params), INTENT(IN) :: p
       INTEGER(C_INT64_T), VALUE :: n_el, n_ion
       TYPE(C_PTR), INTENT(OUT) :: h
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_set_params(h, p) BIND(C)
       IMPORT :: C_INT, C_PTR, tree_gpu_params
       TYPE(C_PTR), VALUE :: h
       TYPE(tree_gpu_params), INTENT(IN) :: p
     END FUNCTION

     ! CALL Force(NS, qel, qion, param, ttime) (main.f90:130, 777, 821)
     INTEGER(C_INT) FUNCTION tree_gpu_force(h, x_el, x_ion, f_el, f_ion, &
          epot_e, epot_i, rdf_ei, rdf_ii) BIND(C)
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: h
       REAL(C_DOUBLE), INTENT(IN) :: x_el(*), x_ion(*)
       REAL(C_DOUBLE), INTENT(OUT) :: f_el(*), f_ion(*), epot_e, epot_i
       TYPE(C_PTR), VALUE :: rdf_ei, rdf_ii   ! C_LOC(int64 array) or C_NULL_PTR
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_set_state(h, x_el, v_el, x_ion, v_ion) BIND(C)
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: h
       REAL(C_DOUBLE), INTENT(IN) :: x_el(*), v_el(*), x_ion(*), v_ion(*)
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_load_state(h, x_el, v_el, f_el, &
          x_ion, v_ion, f_ion) BIND(C)
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: h
       REAL(C_DOUBLE), INTENT(IN) :: x_el(*), v_el(*), f_el(*), x_ion(*), v_ion(*), f_ion(*)
     END FUNCTION

     ! VVerletNotemp1 -> Force -> VVerletNotemp2, nsteps times (main.f90:125-131)
     INTEGER(C_INT) FUNCTION tree_gpu_step(h, dt, nsteps, d) BIND(C)
       IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT32_T, tree_gpu_diag
       TYPE(C_PTR), VALUE :: h
       REAL(C_DOUBLE), VALUE :: dt
       INTEGER(C_INT32_T), VALUE :: nsteps
       TYPE(tree_gpu_diag), INTENT(OUT) :: d
     END FUNCTION

     ! the loop main.f90:123-160 with its Nsamp cadence and per-step RDF
     INTEGER(C_INT) FUNCTION tree_gpu_run(h, dt, nsteps, nsamp, series, &
          series_cap, n_series, rdf_ei, rdf_ii) BIND(C)
       IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT32_T, tree_gpu_sample
       TYPE(C_PTR), VALUE :: h
       REAL(C_DOUBLE), VALUE :: dt
       INTEGER(C_INT32_T), VALUE :: nsteps, nsamp, series_cap
       TYPE(tree_gpu_sample), INTENT(OUT) :: series(*)
       INTEGER(C_INT32_T), INTENT(OUT) :: n_series
       TYPE(C_PTR), VALUE :: rdf_ei, rdf_ii   ! C_LOC(int64 array) or C_NULL_PTR
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_set_graphs(h, enable) BIND(C)
       IMPORT :: C_INT, C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT32_T), VALUE :: enable
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_get_nloop(h, nloop) BIND(C)
       IMPORT :: C_INT, C_PTR, C_INT64_T
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT64_T), INTENT(OUT) :: nloop
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_get_state(h, x_el, v_el, f_el, &
          x_ion, v_ion, f_ion) BIND(C)
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: h
       REAL(C_DOUBLE), INTENT(OUT) :: x_el(*), v_el(*), f_el(*), x_ion(*), v_ion(*), f_ion(*)
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_direct(h, targets, nt, f, epot) BIND(C)
       IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT64_T
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT64_T), INTENT(IN) :: targets(*)
       INTEGER(C_INT64_T), VALUE :: nt
       REAL(C_DOUBLE), INTENT(OUT) :: f(*), epot(*)
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_direct_static(d_x, n_el, n_ion, p, &
          d_targets, nt, d_f, d_epot, stream) BIND(C)
       IMPORT :: C_INT, C_PTR, C_INT64_T, tree_gpu_params
       TYPE(C_PTR), VALUE :: d_x, d_targets, d_f, d_epot, stream  ! device pointers
       INTEGER(C_INT64_T), VALUE :: n_el, n_ion, nt
       TYPE(tree_gpu_params), INTENT(IN) :: p
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_tree_dump(h, species, cap, centre, &
          moments, rcrit, level, skip, pt, n_nodes) BIND(C)
       IMPORT :: C_INT, C_PTR, C_INT32_T, C_INT64_T
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT32_T), VALUE :: species
       INTEGER(C_INT64_T), VALUE :: cap
       TYPE(C_PTR), VALUE :: centre, moments, rcrit, level, skip, pt
       INTEGER(C_INT64_T), INTENT(OUT) :: n_nodes
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_net_dump(h, cap, centre, moments, first, &
          count, level, parent, sorted, n_nodes) BIND(C)
       IMPORT :: C_INT, C_PTR, C_INT64_T
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT64_T), VALUE :: cap
       TYPE(C_PTR), VALUE :: centre, moments, first, count, level, parent, sorted
       INTEGER(C_INT64_T), INTENT(OUT) :: n_nodes
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_set_stream(h, stream) BIND(C)
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: h, stream
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_set_tuning(h, bucket, blocks_per_sm, order) BIND(C)
       IMPORT :: C_INT, C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT32_T), VALUE :: bucket, blocks_per_sm, order
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_set_local_expansion(h, max_ratio) BIND(C)
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: h
       REAL(C_DOUBLE), VALUE :: max_ratio
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_mac_collect(h, theta_lo, theta_hi, rho_lo, &
          rho_hi, max_count, keep, seed, cap, n_total) BIND(C)
       IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT32_T, C_FLOAT, C_INT64_T
       TYPE(C_PTR), VALUE :: h
       REAL(C_DOUBLE), VALUE :: theta_lo, theta_hi, rho_lo, rho_hi
       INTEGER(C_INT32_T), VALUE :: max_count
       REAL(C_FLOAT), VALUE :: keep
       INTEGER(C_INT64_T), VALUE :: seed, cap   ! seed: uint64 in C
       INTEGER(C_INT64_T), INTENT(OUT) :: n_total
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_mac_samples(h, feats, labels, extra, cap, n) BIND(C)
       IMPORT :: C_INT, C_PTR, C_INT64_T
       TYPE(C_PTR), VALUE :: h, feats, labels, extra
       INTEGER(C_INT64_T), VALUE :: cap
       INTEGER(C_INT64_T), INTENT(OUT) :: n
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_mac_clear(h) BIND(C)
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: h
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_mac_train(h, epochs, batch, lr, tau, seed, &
          loss_per_epoch) BIND(C)
       IMPORT :: C_INT, C_PTR, C_INT32_T, C_FLOAT, C_INT64_T
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT32_T), VALUE :: epochs, batch
       REAL(C_FLOAT), VALUE :: lr, tau
       INTEGER(C_INT64_T), VALUE :: seed
       TYPE(C_PTR), VALUE :: loss_per_epoch
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_mac_set_model(h, params, stats) BIND(C)
       IMPORT :: C_INT, C_PTR, C_FLOAT
       TYPE(C_PTR), VALUE :: h
       REAL(C_FLOAT), INTENT(IN) :: params(*), stats(*)
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_mac_get_model(h, params, stats) BIND(C)
       IMPORT :: C_INT, C_PTR, C_FLOAT
       TYPE(C_PTR), VALUE :: h
       REAL(C_FLOAT), INTENT(OUT) :: params(*), stats(*)
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_mac_config(h, eta, rho_lo, rho_hi) BIND(C)
       IMPORT :: C_INT, C_PTR, C_FLOAT
       TYPE(C_PTR), VALUE :: h
       REAL(C_FLOAT), VALUE :: eta, rho_lo, rho_hi
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_mlp_grad(X, y, n, params, tau, grad, loss) BIND(C)
       IMPORT :: C_INT, C_FLOAT, C_INT64_T
       REAL(C_FLOAT), INTENT(IN) :: X(*), y(*), params(*)
       INTEGER(C_INT64_T), VALUE :: n
       REAL(C_FLOAT), VALUE :: tau
       REAL(C_FLOAT), INTENT(OUT) :: grad(*), loss
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_mlp_infer(X, n, params, stats, y) BIND(C)
       IMPORT :: C_INT, C_FLOAT, C_INT64_T
       REAL(C_FLOAT), INTENT(IN) :: X(*), params(*), stats(*)
       INTEGER(C_INT64_T), VALUE :: n
       REAL(C_FLOAT), INTENT(OUT) :: y(*)
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_timings(h, t) BIND(C)
       IMPORT :: C_INT, C_PTR, tree_gpu_timing
       TYPE(C_PTR), VALUE :: h
       TYPE(tree_gpu_timing), INTENT(OUT) :: t
     END FUNCTION

     TYPE(C_PTR) FUNCTION tree_gpu_last_error(h) BIND(C)   ! NUL-terminated C string
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: h
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_destroy(h) BIND(C)
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: h
     END FUNCTION

     TYPE(C_PTR) FUNCTION tree_gpu_version() BIND(C)
       IMPORT :: C_PTR
     END FUNCTION

     ! ensembles of independent clouds; particles cloud-major
     INTEGER(C_INT) FUNCTION tree_gpu_ensemble_create(p, ncloud, n_el, n_ion, h) BIND(C)
       IMPORT :: C_INT, C_INT32_T, C_INT64_T, C_PTR, tree_gpu_params
       TYPE(tree_gpu_params), INTENT(IN) :: p(*)
       INTEGER(C_INT32_T), VALUE :: ncloud
       INTEGER(C_INT64_T), INTENT(IN) :: n_el(*), n_ion(*)
       TYPE(C_PTR), INTENT(OUT) :: h
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_ensemble_set_state(h, x, v) BIND(C)
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: h
       REAL(C_DOUBLE), INTENT(IN) :: x(*), v(*)
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_ensemble_load_state(h, x, v, f) BIND(C)
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: h
       REAL(C_DOUBLE), INTENT(IN) :: x(*), v(*)
       TYPE(C_PTR), VALUE :: f   ! C_LOC(forces) or C_NULL_PTR
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_ensemble_get_state(h, x, v, f) BIND(C)
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: h
       REAL(C_DOUBLE), INTENT(OUT) :: x(*), v(*), f(*)
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_ensemble_sums(h, sums) BIND(C)
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: h
       REAL(C_DOUBLE), INTENT(OUT) :: sums(6, *)
     END FUNCTION

     INTEGER(C_INT) FUNCTION tree_gpu_ensemble_direct(h, cloud, targets, nt, f, epot) BIND(C)
       IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT32_T, C_INT64_T
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT32_T), VALUE :: cloud
       INTEGER(C_INT64_T), INTENT(IN) :: targets(*)
       INTEGER(C_INT64_T), VALUE :: nt
       REAL(C_DOUBLE), INTENT(OUT) :: f(*), epot(*)
     END FUNCTION
  END INTERFACE
END MODULE TREE_GPU_MOD
