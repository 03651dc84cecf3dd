! imago_b200_bind.F90 -- ISO_C_BINDING shim that lets Imago's setupSCF call
! the B200 integral setup (include/imago_intg.h) in place of its
! integral builds.  It is written against the reference's module data and
! HDF5 handles:
!
!    call gaussOverlapOL(...)      -> call b200GaussOverlapOL(...)
!    call gaussOverlapKE(...)      -> call b200GaussOverlapKE(...)
!    call gaussOverlapMV(...)      -> call b200GaussOverlapMV(...)  (rel == 1)
!    call gaussOverlapHamPSCF(...) -> call b200GaussOverlapHamPSCF(...)  (PSCF)
!    call gaussOverlapDM(...)      -> call b200GaussOverlapDM(...)
!    call gaussOverlapMM(...)      -> call b200GaussOverlapMM(...)
!    call gaussKOverlap(...)       -> call b200GaussKOverlap(...)
!    call populateStates           -> call b200PopulateStates
!    call gaussOverlapNP(...)      -> call b200GaussOverlapNP(...)
!    call elecPotGaussOverlap(...) -> call b200ElecPotGaussOverlap(...)
!
! (src/imago/imago.F90:262, 268, 274, 284, 293, 312, 315, 319, 321, 685,
! 705, 709, 714, 716),
! each with the same arguments.
! Each wrapper skips a matrix whose HDF5 "done" attribute is already 1, as
! the reference does, writes the packed valence-valence datasets per
! k-point (and coreValeOL for the overlap) and sets the attribute.
!
! Build line: compile this file with the reference's own sources (it uses
! their modules) and link libimago_b200.so, e.g.
!    h5fc -c imago_b200_bind.F90 && h5fc ... imago_b200_bind.o -limago_b200

module O_ImagoB200

   use, intrinsic :: iso_c_binding
   use O_Kinds
   use HDF5

   implicit none
   private
   public :: b200Setup, b200GaussOverlapOL, b200GaussOverlapKE, &
         & b200GaussOverlapMV, b200GaussOverlapNP, b200ElecPotGaussOverlap, &
         & b200GaussOverlapHamPSCF, b200GaussOverlapDM, b200GaussOverlapMM, &
         & b200GaussKOverlap, b200PopulateStates, b200Cleanup

   type, bind(C) :: imago_system
      real(c_double) :: real_vectors(9)
      real(c_double) :: basis_fn_convg
      real(c_double) :: electro_convg
      integer(c_int) :: num_atom_types
      type(c_ptr) :: type_element
      type(c_ptr) :: type_num_orb_alphas
      type(c_ptr) :: type_alphas
      type(c_ptr) :: type_num_core_fns
      type(c_ptr) :: type_num_vale_fns
      type(c_ptr) :: fn_l
      type(c_ptr) :: fn_coeffs
      integer(c_int) :: num_atom_sites
      type(c_ptr) :: site_type
      type(c_ptr) :: site_pos
      integer(c_int) :: num_pot_types
      type(c_ptr) :: pot_type_element
      type(c_ptr) :: pot_type_nuc_charge
      type(c_ptr) :: pot_type_nuc_alpha
      type(c_ptr) :: pot_type_num_alphas
      type(c_ptr) :: pot_type_alphas
      integer(c_int) :: num_pot_sites
      type(c_ptr) :: pot_site_type
      type(c_ptr) :: pot_site_pos
      integer(c_int) :: num_kpoints
      type(c_ptr) :: kpoints_abc
   end type imago_system

   type, bind(C) :: imago_opts
      integer(c_int) :: device
      type(c_ptr) :: stream
      integer(c_int) :: outputs_on_device
      integer(c_size_t) :: scratch_bytes
   end type imago_opts

   interface
      function imago_intg_create(sys, opts, ctx) &
            & bind(C, name="imago_intg_create") result(st)
         import :: imago_system, imago_opts, c_ptr, c_int
         type(imago_system), intent(in) :: sys
         type(imago_opts), intent(in) :: opts
         type(c_ptr), intent(out) :: ctx
         integer(c_int) :: st
      end function
      function imago_gauss_overlap_ol(ctx, packed, cvre, cvim) &
            & bind(C, name="imago_gauss_overlap_ol") result(st)
         import :: c_ptr, c_int, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: packed(*), cvre(*), cvim(*)
         integer(c_int) :: st
      end function
      function imago_gauss_overlap_ke(ctx, packed) &
            & bind(C, name="imago_gauss_overlap_ke") result(st)
         import :: c_ptr, c_int, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: packed(*)
         integer(c_int) :: st
      end function
      function imago_gauss_overlap_np(ctx, packed) &
            & bind(C, name="imago_gauss_overlap_np") result(st)
         import :: c_ptr, c_int, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: packed(*)
         integer(c_int) :: st
      end function
      function imago_gauss_overlap_mv(ctx, packed) &
            & bind(C, name="imago_gauss_overlap_mv") result(st)
         import :: c_ptr, c_int, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: packed(*)
         integer(c_int) :: st
      end function
      function imago_ham_pscf(ctx, spin, coeffs, rel, packed) &
            & bind(C, name="imago_ham_pscf") result(st)
         import :: c_ptr, c_int, c_double
         type(c_ptr), value :: ctx
         integer(c_int), value :: spin, rel
         real(c_double), intent(in) :: coeffs(*)
         real(c_double), intent(out) :: packed(*)
         integer(c_int) :: st
      end function
      function imago_gauss_overlap_mm(ctx, packed) &
            & bind(C, name="imago_gauss_overlap_mm") result(st)
         import :: c_ptr, c_int, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: packed(*)
         integer(c_int) :: st
      end function
      function imago_gauss_overlap_dm(ctx, center, packed) &
            & bind(C, name="imago_gauss_overlap_dm") result(st)
         import :: c_ptr, c_int, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: center(3)
         real(c_double), intent(out) :: packed(*)
         integer(c_int) :: st
      end function
      function imago_gauss_koverlap(ctx, dk, re, im) &
            & bind(C, name="imago_gauss_koverlap") result(st)
         import :: c_ptr, c_int, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: dk(9)
         real(c_double), intent(out) :: re(*), im(*)
         integer(c_int) :: st
      end function
      function imago_populate_states_sorted(nk, spin, ns, eig, kw, ne, sigma, &
            & srange, slimit, pop, info, sorted, idx) &
            & bind(C, name="imago_populate_states_sorted") result(st)
         import :: c_int, c_double
         integer(c_int), value :: nk, spin, ns
         real(c_double), intent(in) :: eig(*), kw(*)
         real(c_double), value :: ne, sigma, srange, slimit
         real(c_double), intent(out) :: pop(*), info(5), sorted(*)
         integer(c_int), intent(out) :: idx(*)
         integer(c_int) :: st
      end function
      function imago_elec_pot_gauss_overlap(ctx, packed) &
            & bind(C, name="imago_elec_pot_gauss_overlap") result(st)
         import :: c_ptr, c_int, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: packed(*)
         integer(c_int) :: st
      end function
      subroutine imago_intg_destroy(ctx) bind(C, name="imago_intg_destroy")
         import :: c_ptr
         type(c_ptr), value :: ctx
      end subroutine
      function imago_strerror(st) bind(C, name="imago_strerror") result(msg)
         import :: c_int, c_ptr
         integer(c_int), value :: st
         type(c_ptr) :: msg
      end function
   end interface

   type(c_ptr) :: ctx = c_null_ptr
   ! Flattened copies of the module data handed to the C side.
   integer(c_int), allocatable, target :: tElem(:), tNorb(:), tNCore(:), &
         & tNVale(:), fnL(:), sType(:), pElem(:), pNAlpha(:), psType(:)
   real(c_double), allocatable, target :: tAlphas(:), fnC(:), sPos(:), &
         & pZ(:), pNuc(:), pAlphas(:), psPos(:), kAbc(:)

contains

   subroutine fail(st, what)
      integer(c_int), intent(in) :: st
      character(len=*), intent(in) :: what
      write (20,*) what, ' failed with imago status ', st
      stop 'B200 integral setup failed'
   end subroutine fail

   ! Build the imago_system description from the reference's module data
   ! after renormalizeBasis' inputs are read (call after initializeKPoints,
   ! before the integral calls) and stage it on the GPU.
   subroutine b200Setup()
      use O_Lattice, only: realVectors, logBasisFnThresh, logElecThresh
      use O_AtomicTypes, only: numAtomTypes, atomTypes
      use O_AtomicSites, only: numAtomSites, atomSites
      use O_PotTypes, only: numPotTypes, potTypes
      use O_PotSites, only: numPotSites, potSites
      use O_KPoints, only: numKPoints, kPoints
      use O_Constants, only: pi

      type(imago_system) :: sys
      type(imago_opts) :: opts
      integer :: i, j, l, n, nf, nc
      integer(c_int) :: st

      sys%real_vectors = reshape(realVectors, (/9/))
      sys%basis_fn_convg = exp(-logBasisFnThresh)
      sys%electro_convg = exp(-logElecThresh)

      allocate (tElem(numAtomTypes), tNorb(4*numAtomTypes), &
            & tNCore(numAtomTypes), tNVale(numAtomTypes))
      n = 0
      nf = 0
      nc = 0
      do i = 1, numAtomTypes
         tElem(i) = atomTypes(i)%elementID
         tNorb(4*i-3:4*i) = atomTypes(i)%numOrbAlphas(1:4)
         tNCore(i) = atomTypes(i)%numCoreRadialFns
         tNVale(i) = atomTypes(i)%numValeRadialFns
         n = n + atomTypes(i)%numOrbAlphas(1)
         nf = nf + tNCore(i) + tNVale(i)
         do j = 1, tNCore(i)
            nc = nc + atomTypes(i)%numOrbAlphas(atomTypes(i)%coreQN_lList(j)+1)
         enddo
         do j = 1, tNVale(i)
            nc = nc + atomTypes(i)%numOrbAlphas(atomTypes(i)%valeQN_lList(j)+1)
         enddo
      enddo
      allocate (tAlphas(n), fnL(nf), fnC(nc))
      n = 0
      nf = 0
      nc = 0
      do i = 1, numAtomTypes
         l = atomTypes(i)%numOrbAlphas(1)
         tAlphas(n+1:n+l) = atomTypes(i)%alphas(1:l)
         n = n + l
         do j = 1, tNCore(i)
            nf = nf + 1
            fnL(nf) = atomTypes(i)%coreQN_lList(j)
            l = atomTypes(i)%numOrbAlphas(fnL(nf)+1)
            fnC(nc+1:nc+l) = atomTypes(i)%coreRadialFns(1:l,j)
            nc = nc + l
         enddo
         do j = 1, tNVale(i)
            nf = nf + 1
            fnL(nf) = atomTypes(i)%valeQN_lList(j)
            l = atomTypes(i)%numOrbAlphas(fnL(nf)+1)
            fnC(nc+1:nc+l) = atomTypes(i)%valeRadialFns(1:l,j)
            nc = nc + l
         enddo
      enddo
      sys%num_atom_types = numAtomTypes
      sys%type_element = c_loc(tElem)
      sys%type_num_orb_alphas = c_loc(tNorb)
      sys%type_alphas = c_loc(tAlphas)
      sys%type_num_core_fns = c_loc(tNCore)
      sys%type_num_vale_fns = c_loc(tNVale)
      sys%fn_l = c_loc(fnL)
      sys%fn_coeffs = c_loc(fnC)

      allocate (sType(numAtomSites), sPos(3*numAtomSites))
      do i = 1, numAtomSites
         sType(i) = atomSites(i)%atomTypeAssn
         sPos(3*i-2:3*i) = atomSites(i)%cartPos(1:3)
      enddo
      sys%num_atom_sites = numAtomSites
      sys%site_type = c_loc(sType)
      sys%site_pos = c_loc(sPos)

      allocate (pElem(numPotTypes), pZ(numPotTypes), pNuc(numPotTypes), &
            & pNAlpha(numPotTypes))
      n = 0
      do i = 1, numPotTypes
         pElem(i) = potTypes(i)%elementID
         pZ(i) = potTypes(i)%nucCharge
         pNuc(i) = potTypes(i)%nucAlpha
         pNAlpha(i) = potTypes(i)%numAlphas
         n = n + pNAlpha(i)
      enddo
      allocate (pAlphas(n))
      n = 0
      do i = 1, numPotTypes
         pAlphas(n+1:n+pNAlpha(i)) = potTypes(i)%alphas(1:pNAlpha(i))
         n = n + pNAlpha(i)
      enddo
      sys%num_pot_types = numPotTypes
      sys%pot_type_element = c_loc(pElem)
      sys%pot_type_nuc_charge = c_loc(pZ)
      sys%pot_type_nuc_alpha = c_loc(pNuc)
      sys%pot_type_num_alphas = c_loc(pNAlpha)
      sys%pot_type_alphas = c_loc(pAlphas)

      allocate (psType(numPotSites), psPos(3*numPotSites))
      do i = 1, numPotSites
         psType(i) = potSites(i)%potTypeAssn
         psPos(3*i-2:3*i) = potSites(i)%cartPos(1:3)
      enddo
      sys%num_pot_sites = numPotSites
      sys%pot_site_type = c_loc(psType)
      sys%pot_site_pos = c_loc(psPos)

      ! kPoints holds Cartesian bohr^-1 after convertKPointsToXYZ; the C
      ! side takes fractional reciprocal coordinates: k_abc = k . a / 2 pi.
      allocate (kAbc(3*numKPoints))
      do i = 1, numKPoints
         do j = 1, 3
            kAbc(3*(i-1)+j) = sum(kPoints(:,i) * realVectors(:,j)) / (2.0_double*pi)
         enddo
      enddo
      sys%num_kpoints = numKPoints
      sys%kpoints_abc = c_loc(kAbc)

      opts%device = 0
      opts%stream = c_null_ptr
      opts%outputs_on_device = 0
      opts%scratch_bytes = 0
      st = imago_intg_create(sys, opts, ctx)
      if (st /= 0) call fail(st, 'imago_intg_create')
   end subroutine b200Setup

   logical function alreadyDone(aid)
      integer(hid_t), intent(in) :: aid
      integer :: status, hdferr
      integer(hsize_t), dimension(1) :: dims
      dims(1) = 1
      status = 0
      call h5aread_f(aid, H5T_NATIVE_INTEGER, status, dims, hdferr)
      if (hdferr /= 0) stop 'Failed to read integral status.'
      alreadyDone = (status == 1)
   end function alreadyDone

   subroutine markDone(aid)
      integer(hid_t), intent(in) :: aid
      integer :: hdferr
      integer(hsize_t), dimension(1) :: dims
      dims(1) = 1
      call h5awrite_f(aid, H5T_NATIVE_INTEGER, 1, dims, hdferr)
      if (hdferr /= 0) stop 'Failed to record integral success.'
      call h5aclose_f(aid, hdferr)
   end subroutine markDone

   ! Write nk packed matrices [2, nPacked] (complex) or their real parts
   ! (Gamma-only engine, numComponents = 1) to the datasets did(1:nk).
   subroutine writePacked(packed, numComponents, packedVVDims, did, nk, np)
      integer, intent(in) :: numComponents, nk
      integer(hsize_t), intent(in) :: np
      real(c_double), intent(in) :: packed(2, np, nk)
      integer(hsize_t), dimension(2), intent(in) :: packedVVDims
      integer(hid_t), intent(in) :: did(nk)
      integer :: k, hdferr
      do k = 1, nk
         if (numComponents == 2) then
            call h5dwrite_f(did(k), H5T_NATIVE_DOUBLE, packed(:,:,k), &
                  & packedVVDims, hdferr)
         else
            call h5dwrite_f(did(k), H5T_NATIVE_DOUBLE, packed(1:1,:,k), &
                  & packedVVDims, hdferr)
         endif
         if (hdferr /= 0) stop 'Cannot write packed integral matrix.'
      enddo
   end subroutine writePacked

   subroutine b200GaussOverlapOL(numComponents, fullCVDims, packedVVDims, &
         & did, CVdid, aid)
      use O_KPoints, only: numKPoints
      use O_AtomicSites, only: valeDim, coreDim
      use O_Integrals, only: coreValeOL
      integer, intent(in) :: numComponents
      integer(hsize_t), dimension(2), intent(in) :: fullCVDims, packedVVDims
      integer(hid_t), dimension(numKPoints), intent(in) :: did
      integer(hid_t), dimension(numComponents,numKPoints), intent(in) :: CVdid
      integer(hid_t), intent(in) :: aid
      real(c_double), allocatable :: packed(:,:,:), cvre(:,:,:), cvim(:,:,:)
      integer(hsize_t) :: np
      integer :: k, hdferr
      integer(c_int) :: st
      if (alreadyDone(aid)) return
      np = int(valeDim, hsize_t) * (valeDim + 1) / 2
      allocate (packed(2, np, numKPoints))
      allocate (cvre(max(coreDim,1), valeDim, numKPoints))
      allocate (cvim(max(coreDim,1), valeDim, numKPoints))
      st = imago_gauss_overlap_ol(ctx, packed, cvre, cvim)
      if (st /= 0) call fail(st, 'gaussOverlapOL')
      call writePacked(packed, numComponents, packedVVDims, did, numKPoints, np)
      if (coreDim /= 0) then
         do k = 1, numKPoints
            call h5dwrite_f(CVdid(1,k), H5T_NATIVE_DOUBLE, cvre(:,:,k), &
                  & fullCVDims, hdferr)
            if (numComponents == 2) call h5dwrite_f(CVdid(2,k), &
                  & H5T_NATIVE_DOUBLE, cvim(:,:,k), fullCVDims, hdferr)
#ifndef GAMMA
            coreValeOL(:,:,k) = cmplx(cvre(1:coreDim,:,k), cvim(1:coreDim,:,k), &
                  & kind=double)
#endif
         enddo
      endif
      call markDone(aid)
   end subroutine b200GaussOverlapOL

   subroutine b200OneMatrix(which, packedVVDims, did, aid)
      use O_KPoints, only: numKPoints
      use O_AtomicSites, only: valeDim
      integer, intent(in) :: which
      integer(hsize_t), dimension(2), intent(in) :: packedVVDims
      integer(hid_t), dimension(numKPoints), intent(in) :: did
      integer(hid_t), intent(in) :: aid
      real(c_double), allocatable :: packed(:,:,:)
      integer(hsize_t) :: np
      integer(c_int) :: st
      if (alreadyDone(aid)) return
      np = int(valeDim, hsize_t) * (valeDim + 1) / 2
      allocate (packed(2, np, numKPoints))
      if (which == 2) then
         st = imago_gauss_overlap_ke(ctx, packed)
      else if (which == 5) then
         st = imago_gauss_overlap_mv(ctx, packed)
      else
         st = imago_gauss_overlap_np(ctx, packed)
      endif
      if (st /= 0) call fail(st, 'gaussOverlapKE/MV/NP')
      call writePacked(packed, 2, packedVVDims, did, numKPoints, np)
      call markDone(aid)
   end subroutine b200OneMatrix

   subroutine b200GaussOverlapKE(packedVVDims, did, aid)
      use O_KPoints, only: numKPoints
      integer(hsize_t), dimension(2), intent(in) :: packedVVDims
      integer(hid_t), dimension(numKPoints), intent(in) :: did
      integer(hid_t), intent(in) :: aid
      call b200OneMatrix(2, packedVVDims, did, aid)
   end subroutine b200GaussOverlapKE

   subroutine b200GaussOverlapMV(packedVVDims, did, aid)
      use O_KPoints, only: numKPoints
      integer(hsize_t), dimension(2), intent(in) :: packedVVDims
      integer(hid_t), dimension(numKPoints), intent(in) :: did
      integer(hid_t), intent(in) :: aid
      call b200OneMatrix(5, packedVVDims, did, aid)
   end subroutine b200GaussOverlapMV

   subroutine b200GaussOverlapNP(packedVVDims, did, aid)
      use O_KPoints, only: numKPoints
      integer(hsize_t), dimension(2), intent(in) :: packedVVDims
      integer(hid_t), dimension(numKPoints), intent(in) :: did
      integer(hid_t), intent(in) :: aid
      call b200OneMatrix(3, packedVVDims, did, aid)
   end subroutine b200GaussOverlapNP

   subroutine b200ElecPotGaussOverlap(packedVVDims, did, aid)
      use O_KPoints, only: numKPoints
      use O_AtomicSites, only: valeDim
      use O_Potential, only: potDim
      integer(hsize_t), dimension(2), intent(in) :: packedVVDims
      integer(hid_t), dimension(numKPoints,potDim), intent(in) :: did
      integer(hid_t), dimension(potDim), intent(in) :: aid
      real(c_double), allocatable :: packed(:,:,:,:)
      integer(hsize_t) :: np
      integer :: t
      integer(c_int) :: st
      np = int(valeDim, hsize_t) * (valeDim + 1) / 2
      allocate (packed(2, np, numKPoints, potDim))
      st = imago_elec_pot_gauss_overlap(ctx, packed)
      if (st /= 0) call fail(st, 'elecPotGaussOverlap')
      do t = 1, potDim
         if (alreadyDone(aid(t))) cycle
         call writePacked(packed(:,:,:,t), 2, packedVVDims, did(:,t), &
               & numKPoints, np)
         call markDone(aid(t))
      enddo
   end subroutine b200ElecPotGaussOverlap

   ! gaussOverlapHamPSCF + orthoHamPSCF: one packed Hamiltonian per spin
   ! from potCoeffs(potDim, spin), as imago.F90:685 calls it.
   subroutine b200GaussOverlapHamPSCF(did, aid)
      use O_KPoints, only: numKPoints
      use O_AtomicSites, only: valeDim
      use O_Potential, only: rel, spin, potCoeffs
      use O_PSCFIntegralsHDF5, only: packedVVDimsPSCF
      integer(hid_t), dimension(numKPoints,spin), intent(in) :: did
      integer(hid_t), intent(in) :: aid
      real(c_double), allocatable :: packed(:,:,:,:)
      integer(hsize_t) :: np
      integer :: h
      integer(c_int) :: st
      if (alreadyDone(aid)) return
      np = int(valeDim, hsize_t) * (valeDim + 1) / 2
      allocate (packed(2, np, numKPoints, spin))
      st = imago_ham_pscf(ctx, int(spin, c_int), potCoeffs, int(rel, c_int), &
            & packed)
      if (st /= 0) call fail(st, 'gaussOverlapHamPSCF')
      do h = 1, spin
         call writePacked(packed(:,:,:,h), 2, packedVVDimsPSCF, did(:,h), &
               & numKPoints, np)
      enddo
      call markDone(aid)
   end subroutine b200GaussOverlapHamPSCF

   ! gaussOverlapDM / gaussOverlapMM + ortho3Terms: the x, y, z matrices,
   ! written to did(:,1..3) (integrals3Terms.F90:1538-1546).
   subroutine b200ThreeTerms(which, valeValeDims, did, aid)
      use O_KPoints, only: numKPoints
      use O_AtomicSites, only: valeDim
      use O_Input, only: dipoleCenter
      integer, intent(in) :: which
      integer(hsize_t), dimension(2), intent(in) :: valeValeDims
      integer(hid_t), dimension(numKPoints,3), intent(in) :: did
      integer(hid_t), intent(in) :: aid
      real(c_double), allocatable :: packed(:,:,:,:)
      real(c_double) :: center(3)
      integer(hsize_t) :: np
      integer :: j
      integer(c_int) :: st
      if (alreadyDone(aid)) return
      np = int(valeDim, hsize_t) * (valeDim + 1) / 2
      allocate (packed(2, np, numKPoints, 3))
      if (which == 6) then
         center(:) = dipoleCenter(:)
         st = imago_gauss_overlap_dm(ctx, center, packed)
      else
         st = imago_gauss_overlap_mm(ctx, packed)
      endif
      if (st /= 0) call fail(st, 'gaussOverlapDM/MM')
      do j = 1, 3
         call writePacked(packed(:,:,:,j), 2, valeValeDims, did(:,j), &
               & numKPoints, np)
      enddo
      call markDone(aid)
   end subroutine b200ThreeTerms

   subroutine b200GaussOverlapDM(valeValeDims, did, aid)
      use O_KPoints, only: numKPoints
      integer(hsize_t), dimension(2), intent(in) :: valeValeDims
      integer(hid_t), dimension(numKPoints,3), intent(in) :: did
      integer(hid_t), intent(in) :: aid
      call b200ThreeTerms(6, valeValeDims, did, aid)
   end subroutine b200GaussOverlapDM

   subroutine b200GaussOverlapMM(valeValeDims, did, aid)
      use O_KPoints, only: numKPoints
      integer(hsize_t), dimension(2), intent(in) :: valeValeDims
      integer(hid_t), dimension(numKPoints,3), intent(in) :: did
      integer(hid_t), intent(in) :: aid
      call b200ThreeTerms(7, valeValeDims, did, aid)
   end subroutine b200GaussOverlapMM

   ! gaussKOverlap + ortho3Terms(8/9): the overlaps with exp(-i dK_c . r),
   ! dK_c = recipVectors(:,c) / numAxialKPoints(c), written as the full real
   ! (did1) and imaginary (did2) valence planes per k-point and axis, with
   ! the dimensions the reference writes them with
   ! (integrals3Terms.F90:1549-1556).  As in the reference, plusG does not
   ! enter the integrals (integrals3Terms.F90:1287-1298); the caller's
   ! handles decide which group (KOverlap or KOverlapPlusG) is written.
   subroutine b200GaussKOverlap(valeValeDims, did1, did2, aid, plusG)
      use O_KPoints, only: numKPoints, numAxialKPoints
      use O_AtomicSites, only: valeDim
      use O_Lattice, only: recipVectors
      integer(hsize_t), dimension(2), intent(in) :: valeValeDims
      integer(hid_t), dimension(numKPoints,3), intent(in) :: did1, did2
      integer(hid_t), intent(in) :: aid
      real(double), dimension(3,3), intent(in) :: plusG
      real(c_double), allocatable :: re(:,:,:,:), im(:,:,:,:)
      real(c_double) :: dk(3,3)
      integer :: i, j, hdferr
      integer(c_int) :: st
      if (alreadyDone(aid)) return
      do j = 1, 3
         dk(:,j) = recipVectors(:,j) / numAxialKPoints(j)
      enddo
      allocate (re(valeDim, valeDim, numKPoints, 3))
      allocate (im(valeDim, valeDim, numKPoints, 3))
      st = imago_gauss_koverlap(ctx, dk, re, im)
      if (st /= 0) call fail(st, 'gaussKOverlap')
      do j = 1, 3
         do i = 1, numKPoints
            call h5dwrite_f(did1(i,j), H5T_NATIVE_DOUBLE, re(:,:,i,j), &
                  & valeValeDims, hdferr)
            if (hdferr /= 0) stop 'failed to write Koverlap vale vale'
            call h5dwrite_f(did2(i,j), H5T_NATIVE_DOUBLE, im(:,:,i,j), &
                  & valeValeDims, hdferr)
            if (hdferr /= 0) stop 'failed to write Koverlap vale vale'
         enddo
      enddo
      call markDone(aid)
   end subroutine b200GaussKOverlap

   ! populateStates (populate.F90:150-187) through
   ! imago_populate_states_sorted: the eigenvalues are handed over k-point by
   ! k-point, spin by spin, state fastest (the order populateStandard lists
   ! them in), and electronPopulation, occupiedEnergy, occupiedEnergyIndex,
   ! bandGap and gapKindCode are set as the reference sets them.  The module
   ! arrays sortedEnergyEigenValues and indexEnergyEigenValues (1-based
   ! indices) are allocated and filled too, because cleanUpPopulation
   ! (populate.F90:1230-1231), which makeValenceRho calls every iteration,
   ! deallocates them unconditionally.  The XANES core-hole correction
   ! (excitedQN_n /= 0) is not handled: call populateStates then.
   subroutine b200PopulateStates()
      use O_KPoints, only: numKPoints, kPointWeight
      use O_Potential, only: spin
      use O_Input, only: numStates, numElectrons, thermalSigma, &
            & maxThermalRange, fermiSearchLimit
      use O_SecularEquation, only: energyEigenValues
      use O_Populate, only: electronPopulation, occupiedEnergy, &
            & occupiedEnergyIndex, bandGap, gapKindCode, &
            & sortedEnergyEigenValues, indexEnergyEigenValues
      real(c_double), allocatable :: eig(:,:,:)
      integer(c_int), allocatable :: idx(:)
      real(c_double) :: info(5)
      integer :: i, j, n
      integer(c_int) :: st
      n = numStates*numKPoints*spin
      allocate (eig(numStates, spin, numKPoints))
      do i = 1, numKPoints
         do j = 1, spin
            eig(:,j,i) = energyEigenValues(1:numStates,i,j)
         enddo
      enddo
      if (allocated(electronPopulation)) deallocate (electronPopulation)
      if (allocated(sortedEnergyEigenValues)) &
            & deallocate (sortedEnergyEigenValues)
      if (allocated(indexEnergyEigenValues)) deallocate (indexEnergyEigenValues)
      allocate (electronPopulation(n))
      allocate (sortedEnergyEigenValues(n))
      allocate (indexEnergyEigenValues(n))
      allocate (idx(n))
      st = imago_populate_states_sorted(int(numKPoints, c_int), &
            & int(spin, c_int), int(numStates, c_int), eig, kPointWeight, &
            & real(numElectrons, c_double), thermalSigma, maxThermalRange, &
            & fermiSearchLimit, electronPopulation, info, &
            & sortedEnergyEigenValues, idx)
      if (st /= 0) call fail(st, 'populateStates')
      indexEnergyEigenValues(:) = idx(:) + 1
      occupiedEnergy = info(1)
      bandGap = info(2)
      gapKindCode = nint(info(3))
      occupiedEnergyIndex = nint(info(4)) + 1
      deallocate (eig)
      deallocate (idx)
   end subroutine b200PopulateStates

   subroutine b200Cleanup()
      if (c_associated(ctx)) call imago_intg_destroy(ctx)
      ctx = c_null_ptr
   end subroutine b200Cleanup

end module O_ImagoB200
