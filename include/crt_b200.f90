! crt_b200.f90 -- ISO_C_BINDING interface of libcrt_b200.so for the CRTomo /
! CRMod Fortran drivers: one interface per entry point of crt_b200.h, with
! the same names, argument order and meaning.
!
! Conventions:
!  * context and batch handles are TYPE(C_PTR) passed by value;
!  * arrays that are always present are assumed-size dummies of the matching
!    kind (COMPLEX(C_DOUBLE_COMPLEX) for the complex arrays the header passes
!    as double*, in the reference's Fortran layouts: kpot(sanz, eanz,
!    kwnanz), sens(nanz, manz), nrel(elanz+relanz, nk), ...);
!  * arrays the header allows to be NULL are TYPE(C_PTR), VALUE: pass
!    C_LOC(x) or C_NULL_PTR;
!  * scalar outputs are passed by reference; every function returns the
!    reference's errnr (0 = success) unless noted;
!  * uint64_t seeds are INTEGER(C_INT64_T) (same bits).
MODULE crt_b200
  USE, INTRINSIC :: ISO_C_BINDING
  IMPLICIT NONE

  INTEGER(C_INT32_T), PARAMETER :: CRT_B200_ABI_VERSION = 2
  INTEGER(C_INT32_T), PARAMETER :: CRT_PRECOND_JACOBI = 0, CRT_PRECOND_BLOCK = 1, &
       CRT_PRECOND_GNN = 2, CRT_PRECOND_BLOCK_GNN = 3
  INTEGER(C_INT32_T), PARAMETER :: CRT_PREC_FP64 = 0, CRT_PREC_MIXED = 1
  INTEGER(C_INT32_T), PARAMETER :: CRT_FORWARD_AUTO = 0, CRT_FORWARD_DIRECT = 1, CRT_FORWARD_SCHUR = 2

  TYPE, BIND(C) :: crt_mesh
     INTEGER(C_INT32_T) :: sanz, typanz, mb
     TYPE(C_PTR) :: typ, nelanz, selanz      ! [typanz]
     TYPE(C_PTR) :: snr, sx, sy              ! [sanz]
     TYPE(C_PTR) :: nrel                     ! nrel(elanz+relanz, max(selanz))
     TYPE(C_PTR) :: rnr                      ! rnr(relanz)
  END TYPE crt_mesh

  TYPE, BIND(C) :: crt_survey
     INTEGER(C_INT32_T) :: eanz
     TYPE(C_PTR) :: enr
     INTEGER(C_INT32_T) :: nanz
     TYPE(C_PTR) :: strnr, vnr
     INTEGER(C_INT32_T) :: kwnanz, swrtr
     TYPE(C_PTR) :: kwn, kwnwi
     TYPE(C_PTR) :: elbg, relbg, kg          ! precal results, or C_NULL_PTR
     INTEGER(C_INT32_T) :: lsink, nsink
     INTEGER(C_INT32_T) :: rwdanz
     TYPE(C_PTR) :: rwdnr, rwd               ! boundary.dat (lrandb2)
     INTEGER(C_INT32_T) :: lsytop
  END TYPE crt_survey

  TYPE, BIND(C) :: crt_cg_params
     REAL(C_DOUBLE) :: lam, eps
     INTEGER(C_INT32_T) :: ncgmax, ldc, lfpi
     REAL(C_DOUBLE) :: step
     INTEGER(C_INT32_T) :: precond
  END TYPE crt_cg_params

  INTERFACE
     ! -- context --------------------------------------------------------------
     FUNCTION crt_create(device, mesh, survey, precision, errnr) BIND(C, NAME='crt_create')
       IMPORT :: C_PTR, C_INT32_T, crt_mesh, crt_survey
       INTEGER(C_INT32_T), VALUE :: device, precision
       TYPE(crt_mesh), INTENT(IN) :: mesh
       TYPE(crt_survey), INTENT(IN) :: survey
       INTEGER(C_INT32_T), INTENT(OUT) :: errnr
       TYPE(C_PTR) :: crt_create
     END FUNCTION crt_create
     SUBROUTINE crt_destroy(ctx) BIND(C, NAME='crt_destroy')
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: ctx
     END SUBROUTINE crt_destroy
     FUNCTION crt_last_error(ctx) BIND(C, NAME='crt_last_error')
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: ctx
       TYPE(C_PTR) :: crt_last_error            ! NUL-terminated; see crt_error_text
     END FUNCTION crt_last_error
     FUNCTION crt_abi_version() BIND(C, NAME='crt_abi_version')
       IMPORT :: C_INT32_T
       INTEGER(C_INT32_T) :: crt_abi_version
     END FUNCTION crt_abi_version
     FUNCTION crt_set_workspace_limit(ctx, bytes) BIND(C, NAME='crt_set_workspace_limit')
       IMPORT :: C_PTR, C_INT32_T, C_INT64_T
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT64_T), VALUE :: bytes
       INTEGER(C_INT32_T) :: crt_set_workspace_limit
     END FUNCTION crt_set_workspace_limit
     FUNCTION crt_set_refinement(ctx, steps) BIND(C, NAME='crt_set_refinement')
       IMPORT :: C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT32_T), VALUE :: steps
       INTEGER(C_INT32_T) :: crt_set_refinement
     END FUNCTION crt_set_refinement
     FUNCTION crt_set_refinement_tol(ctx, tau) BIND(C, NAME='crt_set_refinement_tol')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_DOUBLE), VALUE :: tau
       INTEGER(C_INT32_T) :: crt_set_refinement_tol
     END FUNCTION crt_set_refinement_tol
     FUNCTION crt_set_forward_form(ctx, form) BIND(C, NAME='crt_set_forward_form')
       IMPORT :: C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT32_T), VALUE :: form      ! CRT_FORWARD_*
       INTEGER(C_INT32_T) :: crt_set_forward_form
     END FUNCTION crt_set_forward_form
     FUNCTION crt_forward_info(ctx, form, nboundary, ninterior, mb_interior) BIND(C, NAME='crt_forward_info')
       IMPORT :: C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: ctx, form, nboundary, ninterior, mb_interior   ! each C_LOC(int) or NULL
       INTEGER(C_INT32_T) :: crt_forward_info
     END FUNCTION crt_forward_info

     ! -- set-up: rwaven, precal ---------------------------------------------------
     FUNCTION crt_rwaven(mesh, eanz, enr, nanz, strnr, vnr, kwnanz, kwn, kwnwi) BIND(C, NAME='crt_rwaven')
       IMPORT :: C_INT32_T, C_DOUBLE, crt_mesh
       TYPE(crt_mesh), INTENT(IN) :: mesh
       INTEGER(C_INT32_T), VALUE :: eanz, nanz
       INTEGER(C_INT32_T), INTENT(IN) :: enr(*), strnr(*), vnr(*)
       INTEGER(C_INT32_T), INTENT(OUT) :: kwnanz
       REAL(C_DOUBLE), INTENT(OUT) :: kwn(*), kwnwi(*)     ! room for 30 (kwnmax)
       INTEGER(C_INT32_T) :: crt_rwaven
     END FUNCTION crt_rwaven
     FUNCTION crt_precal(ctx, elbg, relbg, kg, lbeta, lrandb) BIND(C, NAME='crt_precal')
       IMPORT :: C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: ctx, elbg, relbg, kg   ! Fortran-layout outputs or NULL
       INTEGER(C_INT32_T), INTENT(OUT) :: lbeta, lrandb
       INTEGER(C_INT32_T) :: crt_precal
     END FUNCTION crt_precal

     ! -- forward, potentials, Jacobian --------------------------------------------
     FUNCTION crt_forward(ctx, sigma, ldc, mode, kfak, volt, sigmaa, kpot) BIND(C, NAME='crt_forward')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE_COMPLEX
       TYPE(C_PTR), VALUE :: ctx
       COMPLEX(C_DOUBLE_COMPLEX), INTENT(IN) :: sigma(*)          ! [elanz]
       INTEGER(C_INT32_T), VALUE :: ldc, mode                     ! mode 0 bvolti, 1 bvolt
       TYPE(C_PTR), VALUE :: kfak                                 ! REAL [nanz] or NULL
       COMPLEX(C_DOUBLE_COMPLEX), INTENT(OUT) :: volt(*), sigmaa(*)
       TYPE(C_PTR), VALUE :: kpot                                 ! kpot(sanz, eanz, kwnanz) or NULL
       INTEGER(C_INT32_T) :: crt_forward
     END FUNCTION crt_forward
     FUNCTION crt_potentials(ctx, hpot) BIND(C, NAME='crt_potentials')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE_COMPLEX
       TYPE(C_PTR), VALUE :: ctx
       COMPLEX(C_DOUBLE_COMPLEX), INTENT(OUT) :: hpot(*)          ! hpot(sanz, eanz)
       INTEGER(C_INT32_T) :: crt_potentials
     END FUNCTION crt_potentials
     FUNCTION crt_jacobian(ctx, mode, strom, sens) BIND(C, NAME='crt_jacobian')
       IMPORT :: C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT32_T), VALUE :: mode      ! 0 bsensi, 1 bsendc (real), 2 bsens
       TYPE(C_PTR), VALUE :: strom, sens      ! [nanz] or NULL; sens(nanz, manz) or NULL
       INTEGER(C_INT32_T) :: crt_jacobian
     END FUNCTION crt_jacobian
     FUNCTION crt_set_jacobian(ctx, real_sens, sens) BIND(C, NAME='crt_set_jacobian')
       IMPORT :: C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT32_T), VALUE :: real_sens ! 1: sensdc(nanz, manz) REAL, 0: sens COMPLEX
       TYPE(C_PTR), VALUE :: sens
       INTEGER(C_INT32_T) :: crt_set_jacobian
     END FUNCTION crt_set_jacobian
     FUNCTION crt_voltages_noalloc(kpot, kwnwi, enr, strnr, vnr, sanz, eanz, kwnanz, nanz, swrtr, ldc, mode, &
              kfak, volt, sigmaa, stream) BIND(C, NAME='crt_voltages_noalloc')
       IMPORT :: C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: kpot, kwnwi, enr, strnr, vnr     ! device pointers
       INTEGER(C_INT32_T), VALUE :: sanz, eanz, kwnanz, nanz, swrtr, ldc, mode
       TYPE(C_PTR), VALUE :: kfak, volt, sigmaa, stream       ! device pointers / cudaStream_t
       INTEGER(C_INT32_T) :: crt_voltages_noalloc
     END FUNCTION crt_voltages_noalloc

     ! -- inversion inputs -------------------------------------------------------
     FUNCTION crt_set_configs(ctx, strnr, vnr) BIND(C, NAME='crt_set_configs')
       IMPORT :: C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT32_T), INTENT(IN) :: strnr(*), vnr(*)
       INTEGER(C_INT32_T) :: crt_set_configs
     END FUNCTION crt_set_configs
     FUNCTION crt_set_regularizer(ctx, ltri, nx, nnb, smatm, nachbar) BIND(C, NAME='crt_set_regularizer')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT32_T), VALUE :: ltri, nx, nnb
       REAL(C_DOUBLE), INTENT(IN) :: smatm(*)    ! smatm(manz, 3) or smatm(manz, nnb+1)
       TYPE(C_PTR), VALUE :: nachbar             ! nachbar(manz, nnb+1) or NULL (ltri 0)
       INTEGER(C_INT32_T) :: crt_set_regularizer
     END FUNCTION crt_set_regularizer
     FUNCTION crt_set_data(ctx, dat, wmatd, wdfak) BIND(C, NAME='crt_set_data')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE, C_DOUBLE_COMPLEX
       TYPE(C_PTR), VALUE :: ctx
       COMPLEX(C_DOUBLE_COMPLEX), INTENT(IN) :: dat(*)
       REAL(C_DOUBLE), INTENT(IN) :: wmatd(*)
       TYPE(C_PTR), VALUE :: wdfak               ! INTEGER [nanz] or NULL (= 1)
       INTEGER(C_INT32_T) :: crt_set_data
     END FUNCTION crt_set_data

     ! -- update / lambda search / step ------------------------------------------
     FUNCTION crt_update(ctx, prm, sigmaa, par, dpar, cgfac, cgres, ncg, bdpar) BIND(C, NAME='crt_update')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE_COMPLEX, crt_cg_params
       TYPE(C_PTR), VALUE :: ctx
       TYPE(crt_cg_params), INTENT(IN) :: prm
       TYPE(C_PTR), VALUE :: sigmaa                          ! COMPLEX [nanz] or NULL (last forward)
       COMPLEX(C_DOUBLE_COMPLEX), INTENT(INOUT) :: par(*)    ! [manz]
       TYPE(C_PTR), VALUE :: dpar, cgfac, cgres, ncg, bdpar  ! optional outputs
       INTEGER(C_INT32_T) :: crt_update
     END FUNCTION crt_update
     FUNCTION crt_update_lambdas(ctx, prm, nlam, lams, sigmaa, par, par_out, dpar, ncg, bdpar) &
              BIND(C, NAME='crt_update_lambdas')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE, C_DOUBLE_COMPLEX, crt_cg_params
       TYPE(C_PTR), VALUE :: ctx
       TYPE(crt_cg_params), INTENT(IN) :: prm
       INTEGER(C_INT32_T), VALUE :: nlam                     ! 1 .. 8
       REAL(C_DOUBLE), INTENT(IN) :: lams(*)
       TYPE(C_PTR), VALUE :: sigmaa                          ! COMPLEX [nanz] or NULL
       COMPLEX(C_DOUBLE_COMPLEX), INTENT(IN) :: par(*)       ! [manz]
       COMPLEX(C_DOUBLE_COMPLEX), INTENT(OUT) :: par_out(*)  ! [manz * nlam]
       TYPE(C_PTR), VALUE :: dpar, ncg, bdpar                ! optional outputs
       INTEGER(C_INT32_T) :: crt_update_lambdas
     END FUNCTION crt_update_lambdas
     FUNCTION crt_blam0(ctx, ldc, lfpi, alfx, alfz, lammax) BIND(C, NAME='crt_blam0')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT32_T), VALUE :: ldc, lfpi
       REAL(C_DOUBLE), VALUE :: alfx, alfz
       REAL(C_DOUBLE), INTENT(OUT) :: lammax
       INTEGER(C_INT32_T) :: crt_blam0
     END FUNCTION crt_blam0
     FUNCTION crt_coverage(ctx, part, weight, csens) BIND(C, NAME='crt_coverage')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT32_T), VALUE :: part         ! 0 |J|, 1 |Re J|
       TYPE(C_PTR), VALUE :: weight              ! REAL [nanz] or NULL (sqrt(wmatd wdfak))
       REAL(C_DOUBLE), INTENT(OUT) :: csens(*)   ! [manz]
       INTEGER(C_INT32_T) :: crt_coverage
     END FUNCTION crt_coverage
     FUNCTION crt_gn_step(ctx, prm, par, sigmaa, cgres, ncg, bdpar) BIND(C, NAME='crt_gn_step')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE_COMPLEX, crt_cg_params
       TYPE(C_PTR), VALUE :: ctx
       TYPE(crt_cg_params), INTENT(IN) :: prm
       COMPLEX(C_DOUBLE_COMPLEX), INTENT(INOUT) :: par(*)
       TYPE(C_PTR), VALUE :: sigmaa, cgres, ncg, bdpar       ! optional outputs
       INTEGER(C_INT32_T) :: crt_gn_step
     END FUNCTION crt_gn_step
     FUNCTION crt_set_model(ctx, par) BIND(C, NAME='crt_set_model')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE_COMPLEX
       TYPE(C_PTR), VALUE :: ctx
       COMPLEX(C_DOUBLE_COMPLEX), INTENT(IN) :: par(*)
       INTEGER(C_INT32_T) :: crt_set_model
     END FUNCTION crt_set_model
     FUNCTION crt_gn_step_device(ctx, prm, ncg) BIND(C, NAME='crt_gn_step_device')
       IMPORT :: C_PTR, C_INT32_T, crt_cg_params
       TYPE(C_PTR), VALUE :: ctx
       TYPE(crt_cg_params), INTENT(IN) :: prm
       TYPE(C_PTR), VALUE :: ncg
       INTEGER(C_INT32_T) :: crt_gn_step_device
     END FUNCTION crt_gn_step_device
     FUNCTION crt_get_model(ctx, par) BIND(C, NAME='crt_get_model')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE_COMPLEX
       TYPE(C_PTR), VALUE :: ctx
       COMPLEX(C_DOUBLE_COMPLEX), INTENT(OUT) :: par(*)
       INTEGER(C_INT32_T) :: crt_get_model
     END FUNCTION crt_get_model
     FUNCTION crt_model_backup(ctx, restore) BIND(C, NAME='crt_model_backup')
       IMPORT :: C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT32_T), VALUE :: restore
       INTEGER(C_INT32_T) :: crt_model_backup
     END FUNCTION crt_model_backup
     FUNCTION crt_dmisft(nanz, dat, sigmaa, wmatd, wmatdr, wmatdp, lfpi, lpol, betrms, pharms, npol) &
              BIND(C, NAME='crt_dmisft')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE, C_DOUBLE_COMPLEX
       INTEGER(C_INT32_T), VALUE :: nanz, lfpi, lpol
       COMPLEX(C_DOUBLE_COMPLEX), INTENT(IN) :: dat(*), sigmaa(*)
       REAL(C_DOUBLE), INTENT(IN) :: wmatd(*)
       TYPE(C_PTR), VALUE :: wmatdr, wmatdp, betrms, pharms, npol
       REAL(C_DOUBLE) :: crt_dmisft                         ! nrmsd
     END FUNCTION crt_dmisft

     ! -- diagnostics ---------------------------------------------------------------
     FUNCTION crt_last_timings(ctx, ms7) BIND(C, NAME='crt_last_timings')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_DOUBLE), INTENT(OUT) :: ms7(7)
       INTEGER(C_INT32_T) :: crt_last_timings
     END FUNCTION crt_last_timings
     FUNCTION crt_last_timings_ex(ctx, ms, n) BIND(C, NAME='crt_last_timings_ex')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_DOUBLE), INTENT(OUT) :: ms(*)
       INTEGER(C_INT32_T), VALUE :: n
       INTEGER(C_INT32_T) :: crt_last_timings_ex
     END FUNCTION crt_last_timings_ex
     FUNCTION crt_launch_count(ctx) BIND(C, NAME='crt_launch_count')
       IMPORT :: C_PTR, C_INT64_T
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT64_T) :: crt_launch_count
     END FUNCTION crt_launch_count
     FUNCTION crt_cg_info(ctx, form, block, bandwidth) BIND(C, NAME='crt_cg_info')
       IMPORT :: C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: ctx, form, block, bandwidth
       INTEGER(C_INT32_T) :: crt_cg_info
     END FUNCTION crt_cg_info
     FUNCTION crt_rcm_order(n, xadj, adj, order, bandwidth) BIND(C, NAME='crt_rcm_order')
       IMPORT :: C_PTR, C_INT32_T
       INTEGER(C_INT32_T), VALUE :: n
       INTEGER(C_INT32_T), INTENT(IN) :: xadj(*), adj(*)
       INTEGER(C_INT32_T), INTENT(OUT) :: order(*)
       TYPE(C_PTR), VALUE :: bandwidth
       INTEGER(C_INT32_T) :: crt_rcm_order
     END FUNCTION crt_rcm_order

     ! -- learned preconditioner correction (no reference counterpart) -------------
     FUNCTION crt_gnn_nparam() BIND(C, NAME='crt_gnn_nparam')
       IMPORT :: C_INT32_T
       INTEGER(C_INT32_T) :: crt_gnn_nparam
     END FUNCTION crt_gnn_nparam
     FUNCTION crt_gnn_status(ctx, available, trained, form, nrec, guard_fired) BIND(C, NAME='crt_gnn_status')
       IMPORT :: C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: ctx, available, trained, form, nrec, guard_fired
       INTEGER(C_INT32_T) :: crt_gnn_status
     END FUNCTION crt_gnn_status
     FUNCTION crt_gnn_init(ctx, seed) BIND(C, NAME='crt_gnn_init')
       IMPORT :: C_PTR, C_INT32_T, C_INT64_T
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT64_T), VALUE :: seed
       INTEGER(C_INT32_T) :: crt_gnn_init
     END FUNCTION crt_gnn_init
     FUNCTION crt_gnn_set_weights(ctx, w, n, form) BIND(C, NAME='crt_gnn_set_weights')
       IMPORT :: C_PTR, C_INT32_T, C_FLOAT
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_FLOAT), INTENT(IN) :: w(*)
       INTEGER(C_INT32_T), VALUE :: n, form
       INTEGER(C_INT32_T) :: crt_gnn_set_weights
     END FUNCTION crt_gnn_set_weights
     FUNCTION crt_gnn_get_weights(ctx, w, n, form) BIND(C, NAME='crt_gnn_get_weights')
       IMPORT :: C_PTR, C_INT32_T, C_FLOAT
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_FLOAT), INTENT(OUT) :: w(*)
       INTEGER(C_INT32_T), VALUE :: n
       INTEGER(C_INT32_T), INTENT(OUT) :: form
       INTEGER(C_INT32_T) :: crt_gnn_get_weights
     END FUNCTION crt_gnn_get_weights
     FUNCTION crt_gnn_collect(ctx, prm, base_block, stride, nmax, nrec) BIND(C, NAME='crt_gnn_collect')
       IMPORT :: C_PTR, C_INT32_T, crt_cg_params
       TYPE(C_PTR), VALUE :: ctx
       TYPE(crt_cg_params), INTENT(IN) :: prm
       INTEGER(C_INT32_T), VALUE :: base_block, stride, nmax
       INTEGER(C_INT32_T), INTENT(OUT) :: nrec
       INTEGER(C_INT32_T) :: crt_gnn_collect
     END FUNCTION crt_gnn_collect
     FUNCTION crt_gnn_clear(ctx) BIND(C, NAME='crt_gnn_clear')
       IMPORT :: C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT32_T) :: crt_gnn_clear
     END FUNCTION crt_gnn_clear
     FUNCTION crt_gnn_train(ctx, epochs, batch, lr, seed, loss_hist) BIND(C, NAME='crt_gnn_train')
       IMPORT :: C_PTR, C_INT32_T, C_INT64_T, C_FLOAT
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT32_T), VALUE :: epochs, batch
       REAL(C_FLOAT), VALUE :: lr
       INTEGER(C_INT64_T), VALUE :: seed
       REAL(C_FLOAT), INTENT(OUT) :: loss_hist(*)
       INTEGER(C_INT32_T) :: crt_gnn_train
     END FUNCTION crt_gnn_train
     FUNCTION crt_gnn_record(ctx, idx, x, t, a, nbr, tnorm2) BIND(C, NAME='crt_gnn_record')
       IMPORT :: C_PTR, C_INT32_T, C_FLOAT
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT32_T), VALUE :: idx
       REAL(C_FLOAT), INTENT(OUT) :: x(*), t(*), a(*), tnorm2
       INTEGER(C_INT32_T), INTENT(OUT) :: nbr(*)
       INTEGER(C_INT32_T) :: crt_gnn_record
     END FUNCTION crt_gnn_record
     FUNCTION crt_gnn_record_grad(ctx, idx, grad, loss) BIND(C, NAME='crt_gnn_record_grad')
       IMPORT :: C_PTR, C_INT32_T, C_FLOAT, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT32_T), VALUE :: idx
       REAL(C_FLOAT), INTENT(OUT) :: grad(*)
       REAL(C_DOUBLE), INTENT(OUT) :: loss
       INTEGER(C_INT32_T) :: crt_gnn_record_grad
     END FUNCTION crt_gnn_record_grad

     ! -- batches of independent problems (no reference counterpart) ----------------
     FUNCTION crt_batch_create(ctxs, count, ldc, jacobian_mode, err) BIND(C, NAME='crt_batch_create')
       IMPORT :: C_PTR, C_INT32_T
       TYPE(C_PTR), INTENT(IN) :: ctxs(*)
       INTEGER(C_INT32_T), VALUE :: count, ldc, jacobian_mode
       INTEGER(C_INT32_T), INTENT(OUT) :: err
       TYPE(C_PTR) :: crt_batch_create
     END FUNCTION crt_batch_create
     SUBROUTINE crt_batch_destroy(b) BIND(C, NAME='crt_batch_destroy')
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: b
     END SUBROUTINE crt_batch_destroy
     FUNCTION crt_batch_error(b) BIND(C, NAME='crt_batch_error')
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: b
       TYPE(C_PTR) :: crt_batch_error
     END FUNCTION crt_batch_error
     FUNCTION crt_batch_set_models(b, sigma) BIND(C, NAME='crt_batch_set_models')
       IMPORT :: C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: b
       TYPE(C_PTR), INTENT(IN) :: sigma(*)       ! C_LOC of each instance's COMPLEX sigma
       INTEGER(C_INT32_T) :: crt_batch_set_models
     END FUNCTION crt_batch_set_models
     FUNCTION crt_batch_run(b, ms) BIND(C, NAME='crt_batch_run')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE
       TYPE(C_PTR), VALUE :: b
       REAL(C_DOUBLE), INTENT(OUT) :: ms
       INTEGER(C_INT32_T) :: crt_batch_run
     END FUNCTION crt_batch_run
     FUNCTION crt_batch_status(b, i) BIND(C, NAME='crt_batch_status')
       IMPORT :: C_PTR, C_INT32_T
       TYPE(C_PTR), VALUE :: b
       INTEGER(C_INT32_T), VALUE :: i
       INTEGER(C_INT32_T) :: crt_batch_status
     END FUNCTION crt_batch_status
     FUNCTION crt_batch_results(b, i, volt, sigmaa, sens) BIND(C, NAME='crt_batch_results')
       IMPORT :: C_PTR, C_INT32_T, C_DOUBLE_COMPLEX
       TYPE(C_PTR), VALUE :: b
       INTEGER(C_INT32_T), VALUE :: i
       COMPLEX(C_DOUBLE_COMPLEX), INTENT(OUT) :: volt(*), sigmaa(*)
       TYPE(C_PTR), VALUE :: sens
       INTEGER(C_INT32_T) :: crt_batch_results
     END FUNCTION crt_batch_results
  END INTERFACE

CONTAINS

  ! The message behind the last errnr as a Fortran string (fetxt).
  FUNCTION crt_error_text(ctx) RESULT(txt)
    TYPE(C_PTR), VALUE :: ctx
    CHARACTER(LEN=256) :: txt
    CHARACTER(KIND=C_CHAR), POINTER :: c(:)
    TYPE(C_PTR) :: p
    INTEGER :: i
    txt = ' '
    p = crt_last_error(ctx)
    IF (.NOT. C_ASSOCIATED(p)) RETURN
    CALL C_F_POINTER(p, c, [256])
    DO i = 1, 256
       IF (c(i) == C_NULL_CHAR) EXIT
       txt(i:i) = c(i)
    END DO
  END FUNCTION crt_error_text

END MODULE crt_b200
