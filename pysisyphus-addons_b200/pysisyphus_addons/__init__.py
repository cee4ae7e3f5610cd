"""B200 (sm_100a) implementation of the density-fitting path of pysisyphus-addons.

The public entry points keep the reference's module layout:

* ``pysisyphus_addons.intor.intor``: ``int_schwarz_aux``, ``int_schwarz_bra``
* ``pysisyphus_addons.diabatization.intor``: ``contract_coulomb_densities_2d``,
  ``contract_coulomb_densities_4d``
* ``pysisyphus_addons.std.intor``: ``int_eri2c``, ``int_df1c``, ``int_df2c_mo``

They call ``libpa_b200.so`` (CUDA, FP64) through ctypes; see ``_native``.
``pysisyphus_addons.device`` offers the same path on device-resident torch
tensors.
"""
