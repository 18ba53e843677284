from .transient import main

main()
