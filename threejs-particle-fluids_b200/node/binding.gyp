{
  "targets": [
    {
      "target_name": "pfsim_napi",
      "sources": ["pfsim_napi.c"],
      "include_dirs": ["../../include"],
      "libraries": ["-L<(module_root_dir)/../pfsim", "-lpfsim", "-Wl,-rpath,<(module_root_dir)/../pfsim"],
      "cflags": ["-std=c11", "-O2", "-Wall"]
    }
  ]
}
